// Shared 2D definitions: the grid descriptor, the field handle (four SoA planes) and the
// constants of the step, used by the forward kernels (awcm2d.cu) and the adjoint kernels
// (awcm2d_adjoint.cu).
#pragma once
#include "awcm_common.cuh"

namespace awcm {

constexpr int kMaxLevels = 24;
constexpr int kStages = 3;

struct Grid2 {
    int nx, ny, maxl, pitch, rows, bc_kind;
    double x_min, y_min, dx, dy, gamma;
    double wz_eps;    // WENO-Z epsilon of the face reconstructions (1e-40 as in the reference)
    double wz_delta;  // > 0: tau = sqrt((b0-b2)^2 + wz_delta^2) instead of |b0 - b2| (0 as in the reference)
    const int8_t* bcf;  // kind AWCM_BC_GENERIC: BOUNDARY_CONDITION of every ghosted point (plane layout)
    int wt_i, wt_j;     // kind AWCM_BC_WIND_TUNNEL: the step corner int(0.6/dx), int(0.2/dy)
    Weights W;
    __host__ __device__ __forceinline__ size_t at(int i, int j) const
    {
        return (size_t)(j + kGhost) * pitch + (size_t)(i + kGhost);
    }
    __host__ __device__ __forceinline__ double w(int cnt, int k) const { return W.w[cnt][k + 1]; }
    __host__ __device__ __forceinline__ int D(int lev) const { return 1 << (maxl - lev); }
};

struct Field4 {
    double* p[4];
};


// Adjoint kernel launchers (awcm2d_adjoint.cu, built with FMA contraction: the adjoint is a
// derivative, checked against finite differences, not a bit-exact restatement).
struct AdjStage {
    Grid2 g;
    Field4 qin;        // stage input with its ghost ring filled
    Field4 lam;        // adjoint accumulated into (minus the VJP of the stage residual)
    Field4 nu;         // per-point weight of the residual (zero off the stage mask)
    const uint8_t* m;
    const int8_t* lvl;
    int bit;           // mask bit of the stage
    const uint32_t* xf;
    const unsigned* nxf;
    const uint32_t* yf;
    const unsigned* nyf;
    const uint32_t* crs;
    const unsigned* ncrs;
    const double* ax;  // LF speeds of the stage (per row / per column)
    const double* ay;
};
void adj_launch_stage(const AdjStage& a, int face_blocks, cudaStream_t s);
// RK3 combination adjoints; stage 3 first.  sc: dt/(dx 2^(maxl-lev)) per level.
void adj_launch_rk(int stage, const Grid2& g, size_t plane, const uint8_t* m, const int8_t* lvl, const double* sc,
                   Field4 lam_next, Field4 lam_n, Field4 lam_in, Field4 nu, cudaStream_t s);
void adj_launch_fold(const Grid2& g, Field4 lam, cudaStream_t s);
// Loss 1/2 sum over the mask0 points of (rho - target)^2 (reduced in a fixed order) and its
// gradient seed; target: Ny x Nx doubles on the device; rowsum: Ny doubles scratch.
void adj_launch_seed(const Grid2& g, Field4 q, const uint8_t* m, const double* target, Field4 lam, double* rowsum,
                     double* loss, cudaStream_t s);

}  // namespace awcm
