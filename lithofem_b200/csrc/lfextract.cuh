// Device extraction of the per-mesh data (the reference's extract_asm_data,
// solver/asm_data.inc:99-173, over MFEM's Nedelec space): from a periodic
// tetrahedral mesh (topological vertex ids after identification, the
// element's own vertex coordinates) to the AsmData arrays lfasm_init takes.
//
// Element-local vertex order: ascending topological id, the last two
// swapped where that makes detJ > 0.  Edges and faces are numbered by the
// first occurrence of their key in row order (row = element * 6 + local
// edge, element * 4 + local face): a stable radix sort of the keys, a head
// flag per new key, and a second sort of the runs by their first row.  A
// face's global vertex order is that of its first occurrence; the face
// orientation code is the index of the local-to-global permutation in
// FACE_PERMS.  DOFs: p per edge (reversed on a negative edge), p (p - 1) per
// face (pairs at the face points, permuted by the orientation), the rest
// interior; essential: every DOF of a face that one element alone
// references, with its edges.
#pragma once

#include <cstdint>

namespace lfasm_ex {

__constant__ int c_tet_edges[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
__constant__ int c_tet_faces[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
__constant__ int c_face_perms[6][3] = {{0, 1, 2}, {1, 0, 2}, {1, 2, 0},
                                       {2, 1, 0}, {2, 0, 1}, {0, 2, 1}};
// edges of each local face (the face's boundary edges)
__constant__ int c_face_edges[4][3] = {{3, 4, 5}, {2, 5, 1}, {0, 4, 2}, {1, 3, 0}};

constexpr int EX_ERR_REPEATED = 1;   // an element repeats a vertex
constexpr int EX_ERR_DEGENERATE = 2; // detJ <= 0 after the orientation swap

__device__ __forceinline__ double det3(const double J[9]) {
  return J[0] * (J[4] * J[8] - J[5] * J[7]) - J[1] * (J[3] * J[8] - J[5] * J[6]) +
         J[2] * (J[3] * J[7] - J[4] * J[6]);
}

// local order, Jacobian (row-major, columns x_{c+1} - x_0), inverse
// (adjugate / det), detJ, v0; *err = first failure code, *bad = its element
__global__ void k_ex_local(int ne, const int *__restrict__ tv_in, const double *__restrict__ xv_in,
                           int *__restrict__ tv, double *__restrict__ J9,
                           double *__restrict__ Ji9, double *__restrict__ detJ,
                           double *__restrict__ v0, int *__restrict__ err, int *__restrict__ bad) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int id[4], ord[4] = {0, 1, 2, 3};
  for (int i = 0; i < 4; ++i) id[i] = tv_in[(size_t)e * 4 + i];
  // stable insertion sort of the four ids
  for (int i = 1; i < 4; ++i)
    for (int j = i; j > 0 && id[ord[j - 1]] > id[ord[j]]; --j) {
      const int t = ord[j]; ord[j] = ord[j - 1]; ord[j - 1] = t;
    }
  for (int i = 1; i < 4; ++i)
    if (id[ord[i]] == id[ord[i - 1]]) {
      if (atomicCAS(err, 0, EX_ERR_REPEATED) == 0) *bad = e;
      return;
    }
  double x[4][3];
  for (int i = 0; i < 4; ++i)
    for (int d = 0; d < 3; ++d) x[i][d] = xv_in[((size_t)e * 4 + ord[i]) * 3 + d];
  double J[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) J[r * 3 + c] = x[c + 1][r] - x[0][r];
  double det = det3(J);
  if (det < 0.0) {
    const int t = ord[2]; ord[2] = ord[3]; ord[3] = t;
    for (int d = 0; d < 3; ++d) {
      const double s = x[2][d]; x[2][d] = x[3][d]; x[3][d] = s;
    }
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) J[r * 3 + c] = x[c + 1][r] - x[0][r];
    det = det3(J);
  }
  if (!(det > 0.0)) {
    if (atomicCAS(err, 0, EX_ERR_DEGENERATE) == 0) *bad = e;
    return;
  }
  const double id_ = 1.0 / det;
  double Ji[9];
  Ji[0] = (J[4] * J[8] - J[5] * J[7]) * id_;
  Ji[1] = (J[2] * J[7] - J[1] * J[8]) * id_;
  Ji[2] = (J[1] * J[5] - J[2] * J[4]) * id_;
  Ji[3] = (J[5] * J[6] - J[3] * J[8]) * id_;
  Ji[4] = (J[0] * J[8] - J[2] * J[6]) * id_;
  Ji[5] = (J[2] * J[3] - J[0] * J[5]) * id_;
  Ji[6] = (J[3] * J[7] - J[4] * J[6]) * id_;
  Ji[7] = (J[1] * J[6] - J[0] * J[7]) * id_;
  Ji[8] = (J[0] * J[4] - J[1] * J[3]) * id_;
  for (int i = 0; i < 4; ++i) tv[(size_t)e * 4 + i] = id[ord[i]];
  for (int k = 0; k < 9; ++k) {
    J9[(size_t)e * 9 + k] = J[k];
    Ji9[(size_t)e * 9 + k] = Ji[k];
  }
  detJ[e] = det;
  for (int d = 0; d < 3; ++d) v0[(size_t)e * 3 + d] = x[0][d];
}

// edge keys (min id << 32 | max id) and signs (+1: local order = global)
__global__ void k_ex_edge_keys(int ne, const int *__restrict__ tv,
                               unsigned long long *__restrict__ key, int *__restrict__ row,
                               signed char *__restrict__ sgn) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= (long long)ne * 6) return;
  const int e = (int)(r / 6), le = (int)(r % 6);
  const unsigned a = (unsigned)tv[(size_t)e * 4 + c_tet_edges[le][0]];
  const unsigned b = (unsigned)tv[(size_t)e * 4 + c_tet_edges[le][1]];
  key[r] = a < b ? ((unsigned long long)a << 32 | b) : ((unsigned long long)b << 32 | a);
  row[r] = (int)r;
  sgn[r] = a < b ? 1 : -1;
}

// face keys: the sorted vertex triple, 21 bits each
__global__ void k_ex_face_keys(int ne, const int *__restrict__ tv,
                               unsigned long long *__restrict__ key, int *__restrict__ row) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= (long long)ne * 4) return;
  const int e = (int)(r / 4), f = (int)(r % 4);
  unsigned v[3];
  for (int t = 0; t < 3; ++t) v[t] = (unsigned)tv[(size_t)e * 4 + c_tet_faces[f][t]];
  if (v[0] > v[1]) { const unsigned s = v[0]; v[0] = v[1]; v[1] = s; }
  if (v[1] > v[2]) { const unsigned s = v[1]; v[1] = v[2]; v[2] = s; }
  if (v[0] > v[1]) { const unsigned s = v[0]; v[0] = v[1]; v[1] = s; }
  key[r] = (unsigned long long)v[0] << 42 | (unsigned long long)v[1] << 21 | v[2];
  row[r] = (int)r;
}

// head flags of the sorted keys
__global__ void k_ex_heads(long long n, const unsigned long long *__restrict__ ks,
                           int *__restrict__ head) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  head[i] = (i == 0 || ks[i] != ks[i - 1]) ? 1 : 0;
}

// per run (run = inclusive scan of heads - 1): its first row, its length
__global__ void k_ex_runs(long long n, const int *__restrict__ head, const int *__restrict__ run,
                          const int *__restrict__ rows_s, int *__restrict__ run_first,
                          int *__restrict__ run_len, int *__restrict__ run_idx) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = run[i] - 1;
  if (head[i]) {
    run_first[r] = rows_s[i];  // the stable sort keeps the lowest row first
    run_idx[r] = r;
  }
  atomicAdd(&run_len[r], 1);
}

__global__ void k_ex_rank(int nrun, const int *__restrict__ sorted_run, int *__restrict__ rank) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nrun) rank[sorted_run[j]] = j;
}

// id of every row; first row and multiplicity of every id
__global__ void k_ex_ids(long long n, const int *__restrict__ run, const int *__restrict__ rows_s,
                         const int *__restrict__ rank, const int *__restrict__ run_first,
                         const int *__restrict__ run_len, int *__restrict__ id,
                         int *__restrict__ first_of, int *__restrict__ count_of) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = run[i] - 1, k = rank[r];
  id[rows_s[i]] = k;
  if (i == 0 || run[i - 1] != run[i]) {
    first_of[k] = run_first[r];
    count_of[k] = run_len[r];
  }
}

// face orientation: the permutation from the local vertex order of (e, f)
// to the face's global order (that of its first occurrence)
__global__ void k_ex_face_orient(int ne, const int *__restrict__ tv, const int *__restrict__ fid,
                                 const int *__restrict__ first_of, int *__restrict__ fo,
                                 int *__restrict__ err, int *__restrict__ bad) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= (long long)ne * 4) return;
  const int e = (int)(r / 4), f = (int)(r % 4);
  const int r0 = first_of[fid[r]], e0 = r0 / 4, f0 = r0 % 4;
  int pos[3];
  for (int t = 0; t < 3; ++t) {
    const int v = tv[(size_t)e * 4 + c_tet_faces[f][t]];
    pos[t] = -1;
    for (int j = 0; j < 3; ++j)
      if (tv[(size_t)e0 * 4 + c_tet_faces[f0][j]] == v) pos[t] = j;
  }
  int code = -1;
  for (int c = 0; c < 6; ++c)
    if (c_face_perms[c][0] == pos[0] && c_face_perms[c][1] == pos[1] &&
        c_face_perms[c][2] == pos[2])
      code = c;
  if (code < 0) {
    if (atomicCAS(err, 0, EX_ERR_REPEATED) == 0) *bad = e;
    code = 0;
  }
  fo[r] = code;
}

// DOF map and signs of every element
__global__ void k_ex_dofs(int ne, int p, int nd, int n_edge_dofs, int n_face_dofs,
                          const int *__restrict__ eid, const signed char *__restrict__ esgn,
                          const int *__restrict__ fid, const int *__restrict__ fo,
                          int *__restrict__ dof, double *__restrict__ sign) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int *d = dof + (size_t)e * nd;
  double *s = sign + (size_t)e * nd;
  for (int le = 0; le < 6; ++le) {
    const int g = eid[(size_t)e * 6 + le], sg = esgn[(size_t)e * 6 + le];
    for (int k = 0; k < p; ++k) {
      d[le * p + k] = g * p + (sg > 0 ? k : p - 1 - k);
      s[le * p + k] = sg;
    }
  }
  const int ndof_f = p * (p - 1), npt = ndof_f / 2;
  for (int f = 0; f < 4 && p >= 2; ++f) {
    const int g = fid[(size_t)e * 4 + f], code = fo[(size_t)e * 4 + f];
    for (int i = 0; i < npt; ++i) {
      // face point i of the local order is global point sig(i): the single
      // centroid at p = 2; at p = 3 the points near vertices a, b, c follow
      // their vertex, sig(i) = FACE_PERMS[code][i]
      const int j = p == 2 ? 0 : c_face_perms[code][i];
      for (int t = 0; t < 2; ++t) {
        const int col = 6 * p + f * ndof_f + 2 * i + t;
        d[col] = n_edge_dofs + g * ndof_f + 2 * j + t;
        s[col] = 1.0;
      }
    }
  }
  const int nint = nd - 6 * p - 4 * ndof_f, off = n_edge_dofs + n_face_dofs;
  for (int k = 0; k < nint; ++k) {
    d[nd - nint + k] = off + e * nint + k;
    s[nd - nint + k] = 1.0;
  }
}

// essential flags: the DOFs of every boundary face and of its edges
__global__ void k_ex_ess(int ne, int p, int nd, const int *__restrict__ fid,
                         const int *__restrict__ fcount, const int *__restrict__ dof,
                         int *__restrict__ flag) {
  const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (r >= (long long)ne * 4) return;
  const int e = (int)(r / 4), f = (int)(r % 4);
  if (fcount[fid[r]] != 1) return;
  const int *d = dof + (size_t)e * nd;
  for (int t = 0; t < 3; ++t) {
    const int le = c_face_edges[f][t];
    for (int k = 0; k < p; ++k) flag[d[le * p + k]] = 1;
  }
  const int ndof_f = p * (p - 1);
  for (int k = 0; k < ndof_f; ++k) flag[d[6 * p + f * ndof_f + k]] = 1;
}

__global__ void k_ex_compact(int n, const int *__restrict__ flag, const int *__restrict__ pos,
                             int *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && flag[i]) out[pos[i]] = i;
}

}  // namespace lfasm_ex
