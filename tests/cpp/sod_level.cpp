// C++ host use of the level API (include/bamrex/level.hpp): 1D Sod shock
// tube, 400 cells on [0,1], MUSCL-Hancock / van Leer + HLLC, CFL 0.9, run to
// t = 0.2 with the stop-time clamp; writes "<steps> <time>" and the final
// conserved state (3 x 400 doubles, component-slowest) to argv[1].
#include <cstdio>
#include <vector>

#include "bamrex/level.hpp"

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s out.txt\n", argv[0]);
        return 2;
    }
    const int n = 400;
    const double gamma = 1.4;
    bamrex_box box = { { 0, 0, 0 }, { n - 1, 0, 0 } };
    bamrex_level_desc d = {};
    d.spacedim = 1;
    d.domain = box;
    d.prob_lo[0] = 0.0;
    d.prob_hi[0] = 1.0;
    d.bc_lo[0] = d.bc_hi[0] = BAMREX_BC_TRANSMISSIVE;
    d.boxes = &box;
    d.nboxes = 1;
    d.ngrow = 2;
    d.method = BAMREX_MUSCL_HANCOCK;
    d.cfl = 0.9;
    d.parm = bamrex::make_parm(1, gamma, 1.0, BAMREX_VAN_LEER);
    try {
        bamrex::Level level(d);
        std::vector<double> u(3 * n);
        for (int i = 0; i < n; ++i) {
            const double x = (i + 0.5) / n;
            const bool left = x < 0.5;
            const double rho = left ? 1.0 : 0.125, p = left ? 1.0 : 0.1;
            u[i] = rho;
            u[n + i] = 0.0;
            u[2 * n + i] = p / (gamma - 1);
        }
        level.copyIn(u.data());
        double time = 0.0;
        const int steps = level.run(100000, 0.2, time);
        level.copyOut(u.data());
        level.sync();
        FILE* f = std::fopen(argv[1], "w");
        std::fprintf(f, "%d %.17g\n", steps, time);
        for (double v : u) std::fprintf(f, "%.17g\n", v);
        std::fclose(f);
    } catch (const bamrex::Error& e) {
        std::fprintf(stderr, "bamrex error %d: %s\n", e.status(), e.what());
        return 1;
    }
    return 0;
}
