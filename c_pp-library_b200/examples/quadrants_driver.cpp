// The reference's 2D driver loop (Wavelet/main_2d_euler(quad).cpp:56-350) written against the C++
// mirror classes: the AWCM_2D facade, its field hand-over and the step.  Usage:
//   quadrants_driver <num_levels> <nx_coarse> <t_end> <tol> <cfl>
// Prints one line per output: steps, t, |mask0| of the last step, sum of |mask0|, rho checksum.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "awcm_b200.hpp"

int main(int argc, char** argv)
{
    const int num_levels = argc > 1 ? std::atoi(argv[1]) : 4;
    const int nx_coarse = argc > 2 ? std::atoi(argv[2]) : 9;
    const double t_end = argc > 3 ? std::atof(argv[3]) : 0.02;
    const double tol = argc > 4 ? std::atof(argv[4]) : 1e-3;
    const double cfl = argc > 5 ? std::atof(argv[5]) : 0.4;
    try {
        awcm_b200::AWCM_2D awcm(num_levels, nx_coarse, nx_coarse, 0.0, 1.0, 0.0, 1.0, AWCM_BC_TRANSMISSIVE);
        awcm.Initialize(AWCM_PROBLEM_QUADRANTS, 0.5, 0.5);
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
        for (size_t k = 0; k < q.size(); k += 4) sum += q[k];
        std::printf("steps %d t %.17g mask0 %ld updates %.0f rho_sum %.17g\n", steps, t, awcm.MaskSize(0), upd, sum);
    } catch (const awcm_b200::Error& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
