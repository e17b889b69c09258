// CPU oracle aligner types -- TEST INFRASTRUCTURE ONLY.
#pragma once
#include <cstdint>
#include <vector>

#include "orc_math.hpp"
#include "orc_tree.hpp"

namespace orc {

enum { KIND_ICP = 0, KIND_CT = 1, KIND_CT_DUAL = 2 };
enum { MODE_REF32 = 0, MODE_MIXED = 1, MODE_FP64 = 2 };

// ICPParams_ / CTICPParams_ (kd/icp/tree_aligner_base_.h:12-21, kd/cticp/cticp_.h:14-18)
// plus ICPTerminationCriteriaScore_ (kd/icp/icp_stats_.h:84-102).
struct AlignParams {
  float kernel_threshold;
  float damping;
  float max_error;
  float min_normal_cos;
  int32_t min_good_measurements;
  int32_t max_iterations;
  float velocity_damping;
  int32_t term_crit;
  float d_pert;
  float d_score;
};

// ICPStats_ (kd/icp/icp_stats_.h:10-21)
struct OStats {
  int32_t num_inliers, num_outliers, num_bad, num_err_normal, num_err_fn;
  float chi2, chi2_kernelized, pert_pose_norm, pert_vel_norm;
};

struct OPrior {
  int32_t enabled;
  double X_ref[12];
  double Z[12];
  double info[36];
};

struct OResult {
  int32_t ret;
  int32_t iterations;
  double H[144];
  double b[12];
  double dx[12];
  OStats stats;
  OStats log[64];
};

int align(int kind, int mode, const std::vector<const Tree*>& fixed, const std::vector<Iso<double>>& fixed_X,
          const Tree& moving, const AlignParams& P, const OPrior* prior, double* X12, double* v6, const double* fv6,
          int stats_mode, int num_threads, OResult* out);

bool pose_hessian(const double* H12, double* out36);
void product_caches(const double* X12, const double* Xf12, float* out36);
int align_recorded(int kind, const std::vector<const Tree*>& fixed, const std::vector<Iso<double>>& fixed_X,
                   const Tree& moving, const AlignParams& P, double* X12, double* v6, const double* fv6,
                   OResult* out, std::vector<int32_t>& match, std::vector<int32_t>& status);
void align_replay64(int kind, const std::vector<const Tree*>& fixed, const std::vector<Iso<double>>& fixed_X,
                    const Tree& Mv, const AlignParams& P, double* X12, double* v6, const double* fv6, int iterations,
                    const int32_t* match, const int32_t* status);

void linearize_at(int kind, const Tree& F, const Tree& Mv, const float* caches36, const float* v6, const float* fv6,
                  const AlignParams& P, int stats_mode, int32_t* match_out, int32_t* status_out, double* H_out,
                  double* b_out, OStats* st_out);

template <class T>
void err_jac_vel_A(T& e, T* J, const Iso<T>& Ta, const V3<T>& pa_l, const V3<T>& na_l, const V3<T>& pb_g,
                   const V3<T>& nb_g, const T* va, T dt);
template <class T>
void err_jac_vel_B(T& e, T* J, const Iso<T>& Tb, const V3<T>& pa_g, const V3<T>& na_g, const V3<T>& pb_l,
                   const V3<T>& nb_l, const T* vb, T dt);

}  // namespace orc
