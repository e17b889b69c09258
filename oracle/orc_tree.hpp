// CPU oracle types -- TEST INFRASTRUCTURE ONLY (see orc_math.hpp for the parity status).
#pragma once
#include <cstdint>
#include <vector>

namespace orc {

// TreeGenerator_ PARAMs (kd/tree/tree_generator_.h:18-25) plus the fixed prune incidence
// of the default-constructed IsGoodLeafPredicate_ (kd/tree/tree_predicates_.h:15).
struct TreeParams {
  int32_t propagate_normal;
  int32_t tree_min_good_leaves;
  int32_t leaf_min_points;
  int32_t leaf_max_points;
  float leaf_density;
  float leaf_min_normal_incidence;
  float leaf_eigenvalue_threshold;  // read by the reference, never used
  float leaf_normal_eigenratio;
  float prune_min_normal_incidence;
  int32_t max_level;
};

// Node_ (kd/tree/node_.h:18-48)
struct Node {
  float mean[3];
  float dir[3];
  double dts_mean;
  double dts_cov;
  int64_t start, end;
  int32_t left, right;
};

struct Tree {
  std::vector<Node> nodes;       // BFS order after prune
  std::vector<int32_t> levels;   // depth of each node
  std::vector<int64_t> leaves;   // leaf node indices, BFS order
  std::vector<int64_t> perm;     // final point order: perm[i] = input index at position i
  double ts_start = 0.0;
  // Tree_::root_mean / root_eigenvalues / root_eigenvectors (column-major) as TreeCPU_'s
  // constructor sets them (kd/tree/tree_cpu_.h:72-86), from the root's FP64 decision
  float root_mean[3] = {0.f, 0.f, 0.f};
  float root_eigenvalues[3] = {0.f, 0.f, 0.f};
  float root_eigenvectors[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  int64_t num_points = 0;
  int64_t num_unpruned = 0;
  bool accepted = false;
};

Tree build_tree(const float* xyz, const double* stamps, int64_t n, const TreeParams& P);
// The reference's float build arithmetic (StableAdder_ sums, closed-form eigen, swap
// partition, std::async above parallel_level), for the timed CPU baseline only.
Tree build_tree_ref32(const float* xyz, const double* stamps, int64_t n, const TreeParams& P, int parallel_level);
void jacobi3(const double A[3][3], double ev[3], double V[3][3]);
// floor(v * 2^64) as a 128-bit two's complement integer (hi, lo): the fixed-point
// grid of the per-node moment sums.
void fx_floor_parts(double v, int64_t* hi, uint64_t* lo);

}  // namespace orc
