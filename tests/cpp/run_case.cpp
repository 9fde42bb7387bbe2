// A PIRO-style driver written against include/piro.hpp: runs the equation of
// the case's simindex with the reference's own loop (src/solve.cpp:11-48) and
// writes field 1 to a raw float file.  Built and run by tests/test_gpu_case.py.
#include <cstdio>
#include <vector>

#include "piro.hpp"

int main(int argc, char **argv)
{
    if (argc != 4) {
        std::fprintf(stderr, "usage: run_case <assets_dir> <case.ini> <out.raw>\n");
        return 2;
    }
    try {
        Piro::Case run(argv[1], argv[2]);
        Piro::process solver(run);
        const piro_case_info info = run.info();
        float time = 0.0f;
        int steps = 0;
        while (time < info.totaltime) {
            if (info.simindex == 0) {
                Piro::scalarMatrix UEqn(solver.ddt_r("T") = solver.laplacian("T", "Alpha"));
                UEqn.Solve(time);
            } else {
                Piro::scalarMatrix UEqn(solver.ddt_r("U") = solver.vector("v") & solver.gradient("U"));
                UEqn.Solve(time);
            }
            time += info.timestep;
            ++steps;
        }
        piro_buf f{1, info.n_cells};
        std::vector<float> out((size_t)info.n_cells);
        Piro::check(piro_field_download(run.get(), f, out.data(), info.n_cells), "piro_field_download");
        FILE *fp = std::fopen(argv[3], "wb");
        if (!fp) return 3;
        std::fwrite(out.data(), sizeof(float), out.size(), fp);
        std::fclose(fp);
        std::printf("steps %d\n", steps);
    } catch (const Piro::Error &e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
