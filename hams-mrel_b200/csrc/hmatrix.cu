// hmatrix.cu -- cluster tree, ACA compression and the batched H-matrix
// product of hmatrix.h.
#include <algorithm>
#include <climits>
#include <cmath>

#include "hmatrix.h"

namespace hmat {

// ---------------------------------------------------------------------------
// host: cluster tree and block partition
// ---------------------------------------------------------------------------
namespace {

struct Node {
  int s, e;  // positions s..e (inclusive) in cluster order
  int left = -1, right = -1;
  double c[3];
  double diam;
};

}  // namespace

void build_tree(const double* xyz, int n, Tree& t) {
  t = Tree();
  t.n = n;
  t.perm.resize(n);
  for (int i = 0; i < n; ++i) t.perm[i] = i;
  std::vector<double> w((size_t)3 * n);  // working coordinates, row i = (x, y, z), permuted with perm
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) w[3 * i + d] = xyz[i + (size_t)n * d];
  std::vector<Node> nodes;
  // depth-first with an explicit stack, left child first (SPLIT_CLUSTER_ITERATIVE)
  struct Item {
    int s, e, parent, side;
  };
  std::vector<Item> st{{0, n - 1, -1, 0}};
  while (!st.empty()) {
    Item it = st.back();
    st.pop_back();
    const int ns = it.e - it.s + 1;
    if (ns <= 0) continue;
    const int id = (int)nodes.size();
    nodes.push_back(Node{it.s, it.e});
    if (it.parent >= 0) (it.side == 1 ? nodes[it.parent].left : nodes[it.parent].right) = id;
    double lo[3], hi[3], c[3] = {0, 0, 0};
    for (int d = 0; d < 3; ++d) lo[d] = hi[d] = w[3 * it.s + d];
    for (int i = it.s; i <= it.e; ++i)
      for (int d = 0; d < 3; ++d) {
        const double x = w[3 * i + d];
        if (x < lo[d]) lo[d] = x;
        if (x > hi[d]) hi[d] = x;
        c[d] += x;
      }
    double len[3];
    for (int d = 0; d < 3; ++d) {
      nodes[id].c[d] = c[d] / ns;
      len[d] = hi[d] - lo[d];
    }
    nodes[id].diam = std::sqrt(len[0] * len[0] + len[1] * len[1] + len[2] * len[2]);
    if (ns <= kLeaf) continue;
    int dim = 0;
    if (len[1] > len[dim]) dim = 1;
    if (len[2] > len[dim]) dim = 2;
    const double split = 0.5 * (lo[dim] + hi[dim]);
    int i = it.s, j = it.e;
    while (i <= j) {
      if (w[3 * i + dim] <= split) {
        ++i;
      } else {
        for (int d = 0; d < 3; ++d) std::swap(w[3 * i + d], w[3 * j + d]);
        std::swap(t.perm[i], t.perm[j]);
        --j;
      }
    }
    int left_end = std::max(i - 1, it.s);
    if (left_end >= it.e) left_end = it.e - 1;
    st.push_back({left_end + 1, it.e, id, 2});
    st.push_back({it.s, left_end, id, 1});
  }
  // block partition (BUILD_BLOCK_TREE_ITERATIVE)
  std::vector<int2> bst{{0, 0}};
  while (!bst.empty()) {
    const int2 b = bst.back();
    bst.pop_back();
    const Node &R = nodes[b.x], &C = nodes[b.y];
    const int nr = R.e - R.s + 1, nc = C.e - C.s + 1;
    const double dx = R.c[0] - C.c[0], dy = R.c[1] - C.c[1], dz = R.c[2] - C.c[2];
    const double dist = std::sqrt(dx * dx + dy * dy + dz * dz), dmax = std::max(R.diam, C.diam);
    if (dist > kEta * dmax && nr > 1 && nc > 1) {
      if (nr <= 4 || nc <= 4)
        t.dense.push_back({R.s, nr, C.s, nc});
      else
        t.lowrank.push_back({R.s, nr, C.s, nc});
      continue;
    }
    const bool lr = R.left < 0, lc = C.left < 0;
    if (lr && lc) {
      t.dense.push_back({R.s, nr, C.s, nc});
    } else if (lr) {
      bst.push_back({b.x, C.right});
      bst.push_back({b.x, C.left});
    } else if (lc) {
      bst.push_back({R.right, b.y});
      bst.push_back({R.left, b.y});
    } else {
      bst.push_back({R.right, C.right});
      bst.push_back({R.right, C.left});
      bst.push_back({R.left, C.right});
      bst.push_back({R.left, C.left});
    }
  }
  // leaves in position order and, for each, the blocks covering its rows
  std::vector<int> leaf_of(n, -1);
  std::vector<std::pair<int, int>> lv;
  for (const Node& q : nodes)
    if (q.left < 0) lv.push_back({q.s, q.e - q.s + 1});
  std::sort(lv.begin(), lv.end());
  for (size_t k = 0; k < lv.size(); ++k) {
    t.leaves.push_back({lv[k].first, lv[k].second});
    for (int p = lv[k].first; p < lv[k].first + lv[k].second; ++p) leaf_of[p] = (int)k;
  }
  const int nd = (int)t.dense.size(), nl = (int)t.lowrank.size(), nleaf = (int)t.leaves.size();
  std::vector<std::vector<int>> cover(nleaf);
  auto add = [&](int rs, int nr, int id) {
    for (int k = leaf_of[rs]; k <= leaf_of[rs + nr - 1]; ++k) cover[k].push_back(id);
  };
  for (int d = 0; d < nd; ++d) add(t.dense[d].x, t.dense[d].y, d);
  for (int b = 0; b < nl; ++b) add(t.lowrank[b].x, t.lowrank[b].y, nd + b);
  t.leaf_ptr.assign(1, 0);
  for (int k = 0; k < nleaf; ++k) {
    t.leaf_blk.insert(t.leaf_blk.end(), cover[k].begin(), cover[k].end());
    t.leaf_ptr.push_back((int)t.leaf_blk.size());
  }
  long long off = 0;
  for (int b = 0; b < nl; ++b) {
    t.uv_off.push_back(off);
    off += (long long)kRankMax * (t.lowrank[b].y + t.lowrank[b].w);
  }
  t.uv_total = off;
}

namespace {

template <class T>
int up(T*& dst, const std::vector<T>& src) {
  if (src.empty()) return 0;
  if (cudaMalloc(&dst, src.size() * sizeof(T)) != cudaSuccess) return 1;
  return cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess ? 0 : 1;
}

}  // namespace

int upload(const Tree& t, Dev& d) {
  free_dev(d);
  d.n = t.n;
  d.ndense = (int)t.dense.size();
  d.nlow = (int)t.lowrank.size();
  d.nleaves = (int)t.leaves.size();
  if (up(d.perm, t.perm) || up(d.dense, t.dense) || up(d.lowrank, t.lowrank) || up(d.leaves, t.leaves) ||
      up(d.leaf_ptr, t.leaf_ptr) || up(d.leaf_blk, t.leaf_blk) || up(d.uv_off, t.uv_off))
    return 1;
  if (d.nlow > 0) {
    if (cudaMalloc(&d.rank, sizeof(int) * d.nlow) != cudaSuccess) return 1;
    if (cudaMalloc(&d.w_off, sizeof(long long) * d.nlow) != cudaSuccess) return 1;
    if (cudaMalloc(&d.uv, sizeof(double2) * (size_t)t.uv_total) != cudaSuccess) return 1;
  }
  if (cudaMalloc(&d.ap, sizeof(double2) * (size_t)t.n * t.n) != cudaSuccess) return 1;
  return 0;
}

void free_dev(Dev& d) {
  cudaFree(d.perm);
  cudaFree(d.dense);
  cudaFree(d.lowrank);
  cudaFree(d.leaves);
  cudaFree(d.leaf_ptr);
  cudaFree(d.leaf_blk);
  cudaFree(d.uv_off);
  cudaFree(d.rank);
  cudaFree(d.w_off);
  cudaFree(d.uv);
  cudaFree(d.ap);
  d = Dev();
}

// ---------------------------------------------------------------------------
// device
// ---------------------------------------------------------------------------
namespace {

constexpr int kThreads = 256;
constexpr int kRhsTile = 64;  // right-hand sides per product block
constexpr int kJTile = 16;    // inner-dimension tile of the products

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmac(double2 s, double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, fma(-a.y, b.y, s.x)), fma(a.x, b.y, fma(a.y, b.x, s.y)));
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }

// Ap[i + n j] = A[perm[i] + n perm[j]]: one column of Ap per blockIdx.y
__global__ void k_permute(const double2* __restrict__ A, int n, const int* __restrict__ perm, double2* __restrict__ Ap) {
  const int j = blockIdx.y, i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Ap[i + (size_t)n * j] = A[perm[i] + (size_t)n * perm[j]];
}

// largest value (first index on ties) over the block; every thread gets it
__device__ void block_argmax(double& v, int& idx, double* sv, int* si) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
    if (ov > v || (ov == v && oi < idx)) {
      v = ov;
      idx = oi;
    }
  }
  __syncthreads();
  if (lane == 0) {
    sv[wid] = v;
    si[wid] = idx;
  }
  __syncthreads();
  v = sv[0];
  idx = si[0];
  for (int w = 1; w < kThreads / 32; ++w)
    if (sv[w] > v || (sv[w] == v && si[w] < idx)) {
      v = sv[w];
      idx = si[w];
    }
}

__device__ double block_sum(double v, double* sv) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sv[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < kThreads / 32; ++w) s += sv[w];
  return s;
}

// ACA with partial pivoting of one admissible block per thread block
// (ADD_LOWRANK_BLOCK): U column k = residual column / pivot, VH row k =
// residual row; rank -1 when the block stays dense.
__global__ void __launch_bounds__(kThreads) k_aca(Dev d, double tol) {
  const int bi = blockIdx.x, tid = threadIdx.x;
  const int4 b = d.lowrank[bi];
  const int rs = b.x, nr = b.y, cs = b.z, nc = b.w, n = d.n;
  double2* U = d.uv + d.uv_off[bi];
  double2* VH = U + (size_t)nr * kRankMax;  // row l at VH + l nc
  const double2* Ap = d.ap;
  const int kmax = min(kRankMax, min(nr, nc));
  __shared__ int prow[kRankMax];
  __shared__ double2 urow[kRankMax], vcol[kRankMax], du[kRankMax], dv[kRankMax];
  __shared__ double sv[kThreads / 32];
  __shared__ int si[kThreads / 32];
  __shared__ int stop;
  double frob = 0.0;
  int rank = 0;
  for (int k = 0; k < kmax; ++k) {
    // pivot row: the largest |U(:, k-1)| among the rows not used yet; row 0 first
    int pr = 0;
    if (k > 0) {
      double best = -1.0;
      int bidx = INT_MAX;
      for (int i = tid; i < nr; i += kThreads) {
        bool used = false;
        for (int l = 0; l < k; ++l) used |= prow[l] == i;
        if (used) continue;
        const double a = sqrt(cabs2(U[i + (size_t)nr * (k - 1)]));
        if (a > best) {
          best = a;
          bidx = i;
        }
      }
      block_argmax(best, bidx, sv, si);
      if (bidx == INT_MAX) break;  // every row used
      pr = bidx;
    }
    __syncthreads();
    if (tid == 0) prow[k] = pr;
    if (tid < k) urow[tid] = U[pr + (size_t)nr * tid];
    __syncthreads();
    // residual row, its largest entry
    double best = -1.0;
    int pc = INT_MAX;
    for (int j = tid; j < nc; j += kThreads) {
      double2 v = Ap[(rs + pr) + (size_t)n * (cs + j)];
      for (int l = 0; l < k; ++l) v = csub(v, cmul(urow[l], VH[(size_t)l * nc + j]));
      VH[(size_t)k * nc + j] = v;
      const double a = sqrt(cabs2(v));
      if (a > best) {
        best = a;
        pc = j;
      }
    }
    block_argmax(best, pc, sv, si);
    __syncthreads();
    const double2 pe = VH[(size_t)k * nc + pc];
    if (!(sqrt(cabs2(pe)) >= 1e-30)) break;  // the block is already approximated (or not finite)
    if (tid < k) vcol[tid] = VH[(size_t)tid * nc + pc];
    __syncthreads();
    // residual column / pivot
    const double pd = cabs2(pe);
    const double2 rp = make_double2(pe.x / pd, -pe.y / pd);
    double nu = 0.0, nv = 0.0;
    for (int i = tid; i < nr; i += kThreads) {
      double2 v = Ap[(rs + i) + (size_t)n * (cs + pc)];
      for (int l = 0; l < k; ++l) v = csub(v, cmul(U[i + (size_t)nr * l], vcol[l]));
      v = cmul(v, rp);
      U[i + (size_t)nr * k] = v;
      nu += cabs2(v);
    }
    for (int j = tid; j < nc; j += kThreads) nv += cabs2(VH[(size_t)k * nc + j]);
    nu = block_sum(nu, sv);
    nv = block_sum(nv, sv);
    __syncthreads();
    // <u_l, u_k> and <v_l, v_k> for l < k, one warp per l
    const int lane = tid & 31, wid = tid >> 5;
    for (int l = wid; l < k; l += kThreads / 32) {
      double2 su = make_double2(0.0, 0.0), sw = make_double2(0.0, 0.0);
      for (int i = lane; i < nr; i += 32) {
        const double2 a = U[i + (size_t)nr * l], c = U[i + (size_t)nr * k];
        su = cmac(su, make_double2(a.x, -a.y), c);
      }
      for (int j = lane; j < nc; j += 32) {
        const double2 a = VH[(size_t)l * nc + j], c = VH[(size_t)k * nc + j];
        sw = cmac(sw, make_double2(a.x, -a.y), c);
      }
      for (int o = 16; o; o >>= 1) {
        su.x += __shfl_xor_sync(0xffffffffu, su.x, o);
        su.y += __shfl_xor_sync(0xffffffffu, su.y, o);
        sw.x += __shfl_xor_sync(0xffffffffu, sw.x, o);
        sw.y += __shfl_xor_sync(0xffffffffu, sw.y, o);
      }
      if (lane == 0) {
        du[l] = su;
        dv[l] = sw;
      }
    }
    __syncthreads();
    if (tid == 0) {
      double cross = 0.0;
      for (int l = 0; l < k; ++l) cross += du[l].x * dv[l].x - du[l].y * dv[l].y;
      const double uv = sqrt(nu) * sqrt(nv);
      frob += nu * nv + 2.0 * cross;
      stop = uv < tol * sqrt(fmax(frob, 1e-30));
    }
    __syncthreads();
    rank = k + 1;
    if (stop) break;
  }
  if (tid == 0) d.rank[bi] = (rank == 0 || (long long)rank * (nr + nc) >= (long long)nr * nc) ? -1 : rank;
}

__global__ void k_gather_rows(const double2* __restrict__ X, int n, int nrhs, const int* __restrict__ perm,
                              double2* __restrict__ Xp) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)n * nrhs) return;
  const int i = (int)(e % n);
  const size_t c = e / n;
  Xp[e] = X[perm[i] + (size_t)n * c];
}

__global__ void k_scatter_rows(const double2* __restrict__ Yp, int n, int nrhs, const int* __restrict__ perm,
                               double2* __restrict__ Y) {
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (size_t)n * nrhs) return;
  const int i = (int)(e % n);
  const size_t c = e / n;
  Y[perm[i] + (size_t)n * c] = Yp[e];
}

// W_b (rank x nrhs) = VH_b Xp[block columns, :], one thread block per
// (low-rank block, tile of right-hand sides)
__global__ void __launch_bounds__(kThreads) k_hmv_w(Dev d, const double2* __restrict__ Xp, int nrhs,
                                                    double2* __restrict__ W) {
  const int bi = blockIdx.x, c0 = blockIdx.y * kRhsTile, tid = threadIdx.x;
  const int r = d.rank[bi];
  if (r <= 0) return;
  const int4 b = d.lowrank[bi];
  const int nr = b.y, cs = b.z, nc = b.w, n = d.n;
  const double2* VH = d.uv + d.uv_off[bi] + (size_t)nr * kRankMax;
  double2* Wb = W + d.w_off[bi];
  __shared__ double2 sV[kRankMax][kJTile];
  __shared__ double2 sX[kJTile][kRhsTile + 1];
  const int cc = tid % kRhsTile, l0 = tid / kRhsTile;  // outputs (l0 + 4q, cc)
  constexpr int kQ = (kRankMax + 3) / 4;
  double2 acc[kQ];
#pragma unroll
  for (int q = 0; q < kQ; ++q) acc[q] = make_double2(0.0, 0.0);
  for (int j0 = 0; j0 < nc; j0 += kJTile) {
    const int jn = min(kJTile, nc - j0);
    for (int e = tid; e < r * kJTile; e += kThreads) {
      const int l = e / kJTile, jj = e % kJTile;
      sV[l][jj] = jj < jn ? VH[(size_t)l * nc + j0 + jj] : make_double2(0.0, 0.0);
    }
    for (int e = tid; e < kJTile * kRhsTile; e += kThreads) {
      const int jj = e % kJTile, c = e / kJTile;
      sX[jj][c] = (jj < jn && c0 + c < nrhs) ? Xp[(cs + j0 + jj) + (size_t)n * (c0 + c)] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
      const int l = l0 + 4 * q;
      if (l < r)
        for (int jj = 0; jj < kJTile; ++jj) acc[q] = cmac(acc[q], sV[l][jj], sX[jj][cc]);
    }
    __syncthreads();
  }
  if (c0 + cc < nrhs)
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
      const int l = l0 + 4 * q;
      if (l < r) Wb[l + (size_t)r * (c0 + cc)] = acc[q];
    }
}

// Yp[leaf rows, tile of right-hand sides] = sum over the blocks covering the
// leaf: dense Ap[rows, block columns] Xp[block columns, :], low-rank
// U_b[rows, :] W_b
__global__ void __launch_bounds__(kThreads) k_hmv_leaf(Dev d, const double2* __restrict__ Xp, int nrhs,
                                                       const double2* __restrict__ W, double2* __restrict__ Yp) {
  const int lf = blockIdx.x, c0 = blockIdx.y * kRhsTile, tid = threadIdx.x;
  const int2 leaf = d.leaves[lf];
  const int rs = leaf.x, nr = leaf.y, n = d.n;
  __shared__ double2 sA[kJTile][kLeaf + 1];  // [inner][row]
  __shared__ double2 sX[kJTile][kRhsTile + 1];
  const int cc = tid % kRhsTile, i0 = tid / kRhsTile;  // outputs (i0 + 4q, cc)
  constexpr int kQ = kLeaf / 4;
  double2 acc[kQ];
#pragma unroll
  for (int q = 0; q < kQ; ++q) acc[q] = make_double2(0.0, 0.0);
  for (int p = d.leaf_ptr[lf]; p < d.leaf_ptr[lf + 1]; ++p) {
    const int id = d.leaf_blk[p];
    int4 b;
    int r = -1;
    if (id < d.ndense) {
      b = d.dense[id];
    } else {
      b = d.lowrank[id - d.ndense];
      r = d.rank[id - d.ndense];
    }
    const bool dense = r <= 0;
    // inner dimension: block columns (dense) or the rank (low-rank)
    const int inner = dense ? b.w : r;
    const double2* U = dense ? nullptr : d.uv + d.uv_off[id - d.ndense];
    const double2* Wb = dense ? nullptr : W + d.w_off[id - d.ndense];
    const int ro = rs - b.x;  // leaf rows within the block
    for (int j0 = 0; j0 < inner; j0 += kJTile) {
      const int jn = min(kJTile, inner - j0);
      for (int e = tid; e < kJTile * kLeaf; e += kThreads) {
        const int i = e % kLeaf, jj = e / kLeaf;
        double2 v = make_double2(0.0, 0.0);
        if (i < nr && jj < jn)
          v = dense ? d.ap[(rs + i) + (size_t)n * (b.z + j0 + jj)] : U[(ro + i) + (size_t)b.y * (j0 + jj)];
        sA[jj][i] = v;
      }
      for (int e = tid; e < kJTile * kRhsTile; e += kThreads) {
        const int jj = e % kJTile, c = e / kJTile;
        double2 v = make_double2(0.0, 0.0);
        if (jj < jn && c0 + c < nrhs)
          v = dense ? Xp[(b.z + j0 + jj) + (size_t)n * (c0 + c)] : Wb[(j0 + jj) + (size_t)r * (c0 + c)];
        sX[jj][c] = v;
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < kQ; ++q) {
        const int i = i0 + 4 * q;
        for (int jj = 0; jj < kJTile; ++jj) acc[q] = cmac(acc[q], sA[jj][i], sX[jj][cc]);
      }
      __syncthreads();
    }
  }
  if (c0 + cc < nrhs)
#pragma unroll
    for (int q = 0; q < kQ; ++q) {
      const int i = i0 + 4 * q;
      if (i < nr) Yp[(rs + i) + (size_t)n * (c0 + cc)] = acc[q];
    }
}

}  // namespace

int compress(cudaStream_t st, const double2* A, double tol, Dev& d) {
  if (d.n <= 0) return 0;
  k_permute<<<dim3((d.n + 255) / 256, d.n), 256, 0, st>>>(A, d.n, d.perm, d.ap);
  if (d.nlow > 0) k_aca<<<d.nlow, kThreads, 0, st>>>(d, tol);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

long long product_offsets(cudaStream_t st, const std::vector<int>& hrank, int nrhs, Dev& d,
                          std::vector<long long>& hoff) {
  hoff.assign(hrank.size(), 0);
  long long off = 0;
  for (size_t b = 0; b < hrank.size(); ++b) {
    hoff[b] = off;
    if (hrank[b] > 0) off += (long long)hrank[b] * nrhs;
  }
  if (!hoff.empty()) cudaMemcpyAsync(d.w_off, hoff.data(), hoff.size() * sizeof(long long), cudaMemcpyHostToDevice, st);
  return std::max(off, 1LL);
}

int matvec(cudaStream_t st, const Dev& d, const double2* X, double2* Y, int nrhs, double2* xp, double2* yp,
           double2* w, long long* launches) {
  const size_t tot = (size_t)d.n * nrhs;
  const unsigned g = (unsigned)((tot + 255) / 256), tiles = (unsigned)((nrhs + kRhsTile - 1) / kRhsTile);
  k_gather_rows<<<g, 256, 0, st>>>(X, d.n, nrhs, d.perm, xp);
  if (d.nlow > 0) k_hmv_w<<<dim3(d.nlow, tiles), kThreads, 0, st>>>(d, xp, nrhs, w);
  k_hmv_leaf<<<dim3(d.nleaves, tiles), kThreads, 0, st>>>(d, xp, nrhs, w, yp);
  k_scatter_rows<<<g, 256, 0, st>>>(yp, d.n, nrhs, d.perm, Y);
  *launches += 3 + (d.nlow > 0);
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace hmat
