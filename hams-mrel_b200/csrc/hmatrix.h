// hmatrix.h -- hierarchical-matrix form of the influence matrix for the
// GMRES solver (hmatrix.cu): cluster tree and block partition on the host
// (geometry only, once per context), ACA compression of the admissible
// blocks and the batched H-matrix product on the device (per frequency).
//
// Follows HMatrix.f90: bisection of the panel centres at the midpoint of the
// longest bounding-box side down to 32 panels (SPLIT_CLUSTER_ITERATIVE,
// :236-380), blocks admissible when the centre distance exceeds eta = 2 times
// the larger bounding-box diagonal and both sides have more than one panel
// (BUILD_BLOCK_TREE_ITERATIVE, :390-497), ACA with partial pivoting to a
// relative tolerance (1e-4) and rank 50 (ADD_LOWRANK_BLOCK, :560-748), blocks
// of four rows or columns or less, and blocks the ACA cannot compress, kept
// dense.  The product (HMATVEC, :760-820) runs over all right-hand sides at
// once, one thread block per leaf row cluster summing every block that covers
// its rows, so no two blocks write the same output.
//
// The ACA's stopping test uses the exact Frobenius norm of the approximation
// so far, ||S_k||^2 = ||S_k-1||^2 + ||u_k||^2 ||v_k||^2
// + 2 Re sum_l<k <u_l, u_k> <v_l, v_k>; the reference's running sum
// (:696-707) adds products of real parts over the row count instead, so the
// ranks it picks can differ by a few.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace hmat {

constexpr int kLeaf = 32;      // panels per leaf cluster (NLEAF_DEFAULT)
constexpr double kEta = 2.0;   // admissibility (ETA_DEFAULT)
constexpr int kRankMax = 50;   // ACA rank limit (RANK_MAX)
constexpr double kAcaTol = 1e-4;  // ACA tolerance (ACA_TOL)

// Block partition of the permuted matrix (cluster order).
struct Tree {
  int n = 0;
  std::vector<int> perm;             // cluster position -> panel
  std::vector<int4> dense;           // (row start, rows, column start, columns)
  std::vector<int4> lowrank;         // admissible blocks for the ACA
  std::vector<int2> leaves;          // leaf row clusters (start, rows)
  std::vector<int> leaf_ptr;         // CSR over leaves: blocks whose rows cover the leaf
  std::vector<int> leaf_blk;         // block id: dense d as d, low-rank b as ndense + b
  std::vector<long long> uv_off;     // low-rank block b: U (rows x kRankMax) then VH (kRankMax x columns)
  long long uv_total = 0;
};

// Cluster tree and block partition from the panel centres xyz (n x 3,
// column-major).
void build_tree(const double* xyz, int n, Tree& t);

// Device side of a Tree plus the per-frequency data.
struct Dev {
  int n = 0, ndense = 0, nlow = 0, nleaves = 0;
  int* perm = nullptr;
  int4* dense = nullptr;
  int4* lowrank = nullptr;
  int2* leaves = nullptr;
  int* leaf_ptr = nullptr;
  int* leaf_blk = nullptr;
  long long* uv_off = nullptr;
  int* rank = nullptr;        // per low-rank block after the ACA; -1: kept dense
  long long* w_off = nullptr; // per low-rank block: offset of its rank x nrhs product in the work array
  double2* uv = nullptr;      // factor store
  double2* ap = nullptr;      // the matrix in cluster order (n x n)
};

// Upload a tree (device buffers allocated here; free with free_dev).
int upload(const Tree& t, Dev& d);
void free_dev(Dev& d);

// Per frequency: permute A (n x n, column-major) into d.ap and compress the
// admissible blocks; tol is the ACA's relative tolerance.  Returns 0 or 1 on
// a launch error.  After it, d.rank holds the ranks (device).
int compress(cudaStream_t st, const double2* A, double tol, Dev& d);

// Offsets of the per-block products for nrhs right-hand sides from the ranks
// (host copy hrank): fills d.w_off (device) and returns the work size in
// double2 elements.
long long product_offsets(cudaStream_t st, const std::vector<int>& hrank, int nrhs, Dev& d,
                          std::vector<long long>& hoff);

// Y (n x nrhs) = H X (n x nrhs), both column-major with leading dimension n;
// xp, yp (n x nrhs) and w (product_offsets elements) are work arrays.
// Returns 0 or 1 on a launch error; *launches counts the kernels.
int matvec(cudaStream_t st, const Dev& d, const double2* X, double2* Y, int nrhs, double2* xp, double2* yp,
           double2* w, long long* launches);

}  // namespace hmat
