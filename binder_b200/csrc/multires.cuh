// The multi-resolution step of BINDER/FastRegistration.py on the device: move_resolution
// (:550-650) followed by the Registration set-up that run() performs for the new level
// (:443-486), without host copies of the fields, bins or prior eigenvalues.
#pragma once

#include "engine.cuh"

namespace binder {

struct PyramidConfig {
    int nx, ny, nz;      // full-resolution fixed (voxel) grid; nz == 1 for an image
    int nxn, nyn, nzn;   // full-resolution moving (node) grid
    double voxel_size[3], node_size[3];  // voxels_voxel_size, nodes_voxel_size
    double gamma_init;                   // `gamma` of FastRegistration
    int finite_difference_order;
    int increase_gamma_at_ds;            // increase_gamma_at_DS_resolution
    int upsample_in_frequency_domain;
    int spline_order;
};

// What move_resolution computed for a level (FastRegistration attributes of the same names).
struct LevelInfo {
    int voxels_shape[3], nodes_shape[3];
    double gamma[3];
    double voxel_size[3], node_size[3];  // current_voxels_voxel_size, current_nodes_voxel_size
    double non_zero_voxels;
};

class Pyramid {
  public:
    // Full-resolution bins (int32, validated against K / L when a level is set up) and voxel
    // positions in node space (AoS [V][N], FP64; null for the identity grid).  Pointers may be
    // host or device memory; the pyramid keeps device copies.
    Pyramid(const PyramidConfig &c, const int *binned_voxels, const int *binned_nodes,
            const double *voxel_pos);
    ~Pyramid();
    Pyramid(const Pyramid &) = delete;
    Pyramid &operator=(const Pyramid &) = delete;

    // move_resolution(res) and the new level's Registration: the deformation comes from `prev`
    // (a registration at resolution prev_res, which must be idle) or, when prev is null, from
    // the full-resolution voxel positions (resolution 1, as FastRegistration starts).  theta
    // [K][L] may be host or device memory, or null to carry prev's over.
    Registration *level(int res, const Registration *prev, int prev_res, double alpha,
                        const float *theta, int K, int L, LevelInfo *info);

  private:
    PyramidConfig c_;
    int N_;
    cudaStream_t s_ = 0;
    int *u_ = nullptr, *v_ = nullptr;  // full-resolution bins
    double *pos_ = nullptr;            // full-resolution voxel positions or null (identity)
};

}  // namespace binder
