// Jacobian determinants and topology correction (FP64), BINDER/src/cpu/utils.cpp:100-345 and
// BINDER/src/cpu/topology_correction_3D.cpp:17-607.
#pragma once

#include "common.cuh"

namespace binder {

struct JacStats {
    double jmin, jmax;
    long long below, above, negative;
};

// averaged 8-corner Jacobian of an AoS [V][3] field (FP64) -> J [V]
void jacobian3d_device(const double *field_aos, int nx, int ny, int nz, const double vs[3],
                       double *J, cudaStream_t s);

// 2D: the 4-corner Jacobian (BINDER/src/cpu/utils.cpp:10-98) of an AoS [nx][ny][2] field, FP64
void jacobian2d_device(const double *field_aos, int nx, int ny, const double vs[2], double *J,
                       cudaStream_t s);
// the same from host memory into host memory (device buffers from the pool, own stream)
void jacobian2d(const double *field_host, int nx, int ny, const double vs[2], double *J_host);

// The same determinants from a host AoS field into host J, staged through a fixed array in the
// library's device image instead of allocated buffers (grids up to kJacobianNoAllocMaxVoxels).
// Runs on the legacy default stream of the current device and returns when J is on the host.
// Calls that overlap in time on one device share the array and race.  stats may be NULL; its
// `below` / `above` count J < 0 / J > 0.
constexpr long kJacobianNoAllocMaxVoxels = 1L << 19;
void jacobian3d_noalloc(const double *field_host, int nx, int ny, int nz, const double vs[3],
                        double *J_host, JacStats *stats);

// full correction on a host AoS field in grid units (in place)
struct TopologyResult {
    int outer_iterations;
    int inner_iterations;
    long long below_before, above_before, below_after, above_after;
    unsigned flags;
};
TopologyResult topology_correct_3d(double *field_aos_host, double e1, double e2, int max_outer,
                                   int max_inner, const double vs[3], int nx, int ny, int nz,
                                   cudaStream_t s);
// BINDER/src/cpu/topology_correction_2D.cpp:17-163 on a host AoS [nx][ny][2] field (in place)
TopologyResult topology_correct_2d(double *field_aos_host, double e1, double e2, int max_outer,
                                   int max_inner, const double vs[2], int nx, int ny,
                                   cudaStream_t s);
// either of the two (nz == 1: an image with two components)
TopologyResult topology_correct(double *field_aos_host, double e1, double e2, int max_outer,
                                int max_inner, const double vs[3], int nx, int ny, int nz,
                                cudaStream_t s);

// Device buffers of the correction for one grid (positions, gradients, corner Jacobians, Poisson
// work space), reusable across calls.  Positions are SoA [N][V] in physical units, N = 3, or 2
// for an image (nz == 1; vs[2] is then unused).  The buffers
// come from the stream-ordered pool on stream `s`, which must outlive the workspace.
class TopologyWorkspace {
  public:
    TopologyWorkspace(int nx, int ny, int nz, cudaStream_t s);
    ~TopologyWorkspace();
    TopologyWorkspace(const TopologyWorkspace &) = delete;
    TopologyWorkspace &operator=(const TopologyWorkspace &) = delete;
    double *positions();
    // grid-unit FP32 SoA field <-> the workspace's FP64 physical positions
    void load_float_grid(const float *d_soa, const double vs[3], cudaStream_t s);
    void store_float_grid(float *d_soa, const double vs[3], cudaStream_t s);
    TopologyResult run(double e1, double e2, int max_outer, int max_inner, const double vs[3],
                       cudaStream_t s);

  private:
    TopologyResult run2d(double e1, double e2, int max_outer, int max_inner, const double vs[3],
                         cudaStream_t s);
    struct Impl;
    Impl *impl_;
};

}  // namespace binder
