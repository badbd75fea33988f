// The reference's 1D driver loop (Wavelet/main_1d_euler.cpp:61-260) written against the C++
// mirror classes: the AWCM_1D facade, its field hand-over and the step.  Usage:
//   sod_driver <num_levels> <nx_coarse> <t_end> <tol> <cfl> [passes|generic]
// Sod tube on cell-centred nodes of [0,1], interface 0.5.  Prints steps, t, |mask0| of the last
// step, the sum of |mask0| over the steps and a density checksum.  With "passes", the first
// PrepareEuler is also done pass by pass through AWCM_MANAGER_1D and the facade's wavelet calls
// (Wavelet/AWCM_1D.h:86-120, the mask copies through the host) on a second instance, and the
// masks, levels and field are compared with the one-call PrepareEuler ("passes equal 1").  With
// "generic", the ghost fills use the enum-driven BOUNDARY_MANAGER_1D<T> with zero-order
// extrapolation at every ghost cell, which is the transmissive manager's fill.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "awcm_b200.hpp"

using awcm_b200::AWCM_1D;
using awcm_b200::AWCM_MANAGER_1D;

static bool prepare_by_passes_matches(int L, int nxc, double x0, double x1, double tol)
{
    const double left[3] = {1.0, 0.0, 1.0}, right[3] = {0.125, 0.0, 0.1};
    AWCM_1D one(L, nxc, x0, x1), passes(L, nxc, x0, x1);
    one.InitializeRiemann(0.5, left, right);
    passes.InitializeRiemann(0.5, left, right);
    one.PrepareEuler(tol);
    const int w = passes.Nx() + 6;
    std::vector<uint8_t> m(5 * (size_t)w);
    auto copy_mask = [&](int from_id, int to_id) {  // the reference's whole-field mask copies
        awcm_b200::check(awcm1d_batch_get_masks(passes.handle(), 0, m.data()), "get_masks");
        const int pf = from_id == 4 ? 0 : from_id + 1, pt = to_id == 4 ? 0 : to_id + 1;
        std::memcpy(&m[(size_t)pt * w], &m[(size_t)pf * w], (size_t)w);
        awcm_b200::check(awcm1d_batch_set_masks(passes.handle(), 0, m.data()), "set_masks");
    };
    copy_mask(0, 4);  // mask_temp = mask0
    passes.ForwardWaveletTransformEuler(tol);
    passes.BadingBoundary(0);
    AWCM_MANAGER_1D::AddAdjacentZone(passes, 0);
    AWCM_MANAGER_1D::CheckReconstruction(passes, 0);
    for (int k = 1; k <= 3; ++k) {
        copy_mask(k - 1, k);
        AWCM_MANAGER_1D::ComputeLevel(passes, k - 1, k - 1);
        AWCM_MANAGER_1D::AddAdjacentZone(passes, k);
        AWCM_MANAGER_1D::AddPointForDifferentiation(passes, k, k - 1);
        AWCM_MANAGER_1D::CheckReconstruction(passes, k);
    }
    AWCM_MANAGER_1D::ComputeLevel(passes, 3, 3);
    passes.InverseWaveletTransformEuler(3);
    passes.InterpolateEuler(4, 3);
    bool same = one.GetField() == passes.GetField();
    for (int id = 0; id <= 4; ++id) same = same && one.Mask(id) == passes.Mask(id);
    for (int l = 0; l <= 3; ++l) same = same && one.Level(l) == passes.Level(l);
    return same;
}

int main(int argc, char** argv)
{
    const int num_levels = argc > 1 ? std::atoi(argv[1]) : 7;
    const int nx_coarse = argc > 2 ? std::atoi(argv[2]) : 17;
    const double t_end = argc > 3 ? std::atof(argv[3]) : 0.2;
    const double tol = argc > 4 ? std::atof(argv[4]) : 1e-4;
    const double cfl = argc > 5 ? std::atof(argv[5]) : 0.5;
    const bool passes = argc > 6 && std::strcmp(argv[6], "passes") == 0;
    const bool generic = argc > 6 && std::strcmp(argv[6], "generic") == 0;
    try {
        const int nx = (nx_coarse - 1) * (1 << (num_levels - 1)) + 1;
        const double x0 = 0.5 / nx, x1 = 1 - 0.5 / nx;
        if (passes) std::printf("passes equal %d\n", prepare_by_passes_matches(num_levels, nx_coarse, x0, x1, tol) ? 1 : 0);
        AWCM_1D awcm(num_levels, nx_coarse, x0, x1);
        const double left[3] = {1.0, 0.0, 1.0}, right[3] = {0.125, 0.0, 0.1};
        awcm.InitializeRiemann(0.5, left, right);
        if (generic) {
            const std::vector<int> bc((size_t)nx + 6, awcm_b200::EXTRAPOLATION_ZERO_ORDER);
            awcm_b200::BOUNDARY_MANAGER_1D<>(bc).SetBoundaryCondition(awcm);
        }
        double t = 0, upd = 0;
        int steps = 0;
        while (true) {
            bool do_print = false;
            const double dt = awcm.Step(tol, cfl, t, t_end, &do_print);
            t += dt;
            upd += (double)awcm.MaskSize(0);
            ++steps;
            if (t >= t_end) break;
        }
        const std::vector<double> q = awcm.GetField();
        double sum = 0;
        for (size_t k = 0; k < q.size(); k += 3) sum += q[k];
        std::printf("steps %d t %.17g mask0 %ld updates %.0f rho_sum %.17g\n", steps, t, awcm.MaskSize(0), upd, sum);
    } catch (const awcm_b200::Error& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
