// The reference's text outputs and experiment reports written by one program that builds
// against either header set: the C++ adapter (include/amg_b200/amg_b200.hpp, default) or,
// with -DAMG_REFERENCE_BUILD, the reference's own headers and objects (src/variables.cpp,
// include/params.h).  tests/test_cpp_reports.py builds both and compares the files.
//
//   reports_main <workdir>     (the working directory must be <workdir>: the reports are
//                               written to the current directory, as the reference does)
// reads parameters.dat; writes printParameters' banner to stdout, and vec.txt (save_vec),
// rhs.txt (save_rhs of random_rhs with seed 7, twice: the generator is seeded once),
// metadata_*.dat and results_*.out (saveParameters).
#include <cstdio>
#include <string>
#include <vector>

#ifdef AMG_REFERENCE_BUILD
#include "params.h"
#include "variables.h"
#else
#include "amg_b200/amg_b200.hpp"
#endif

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <workdir>\n", argv[0]);
        return 2;
    }
    const std::string wd = argv[1];
    readParameters(wd + "/parameters.dat");
    mass::m0 = -0.25;
    AMGV::cycle = 1;
    AMGV::nu1 = 1;
    AMGV::Nit = 2;
    printParameters();
    save_vec(std::vector<double>{1.0, -2.5e-11, 3.0e7}, "vec.txt");
    std::vector<std::vector<std::complex<double>>> v(LV::Ntot, std::vector<std::complex<double>>(2, 0));
    random_rhs(v, 7);
    save_rhs(v, "rhs1.txt");
    random_rhs(v, 7);
    save_rhs(v, "rhs2.txt");
    double it[3] = {5.0, 6.5, 7.25}, dit[3] = {0.5, 0.25, 0.125}, t[3] = {1.5, 2.5e-3, 3.0}, dt[3] = {0.1, 0.2, 0.3};
    saveParameters(it, dit, t, dt, 3, 17);
    return 0;
}
