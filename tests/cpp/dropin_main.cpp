// A reference-style driver built against include/amg_b200/amg_b200.hpp instead of the
// reference's headers: the same calls its main and its Tests class make
// (src/main.cpp:54-130, src/tests.cpp:67-82), plus the per-level operations of Level and
// AlgebraicMG.  Compiled and run by tests/test_cpp_dropin.py; NS, NT and LEVELS come from
// the compile line as they come from config.h in the reference.
//
//   dropin_main <workdir>
// reads  parameters.dat, gauge.ctxt ("x t mu re im"), rhs.rhs ("x t spin re im"), m0.txt,
//        probe_l<l>.bin (complex128 [N_l][DOF_l])
// writes x.bin, x_sap.bin, x_gmres.bin, x_cg.bin, x_bicg.bin, dphi.bin, ddagphi.bin, dop_l<l>.bin, pt_l0.bin, ppt_l0.bin, sap_l0.bin,
//        gmres_l<L-1>.bin, cycle0_rhs.bin (complex128) and results.txt
#include <cstdio>

#include "amg_b200/amg_b200.hpp"

static void dump(const std::string& path, const spinor& s) {
    std::vector<c_double> f = amg_b200::flatten(s);
    std::ofstream o(path, std::ios::binary);
    o.write(reinterpret_cast<const char*>(f.data()), (std::streamsize)(f.size() * sizeof(c_double)));
}

static bool load(const std::string& path, spinor& s) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return false;
    std::vector<c_double> f(s.size() * s[0].size());
    in.read(reinterpret_cast<char*>(f.data()), (std::streamsize)(f.size() * sizeof(c_double)));
    amg_b200::unflatten(f, s);
    return true;
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <workdir>\n", argv[0]);
        return 2;
    }
    const std::string wd = argv[1];
    try {
        readParameters(wd + "/parameters.dat");
        AMGV::cycle = 1;
        AMGV::Nit = 0;
        AMGV::SAP_test_vectors_iterations = 4;
        double m0 = 0;
        std::ifstream(wd + "/m0.txt") >> m0;

        GaugeConf GConf(LV::Nx, LV::Nt);
        GConf.read_conf(wd + "/gauge.ctxt");
        const spinor x0(LevelV::Nsites[0], c_vector(LevelV::DOF[0], 0));
        spinor rhs(LevelV::Nsites[0], c_vector(LevelV::DOF[0], 0));
        read_rhs(rhs, wd + "/rhs.rhs");

        std::ofstream res(wd + "/results.txt");
        // Tests::fgmresAMG (src/tests.cpp:67-82)
        spinor x(LevelV::Nsites[0], c_vector(LevelV::DOF[0], 0));
        FGMRES_AMG solver(LV::Ntot, 2, FGMRESV::fgmres_restart_length, FGMRESV::fgmres_restarts,
                          FGMRESV::fgmres_tolerance, GConf, m0);
        const int it = solver.fgmres(rhs, x0, x, true, true);
        dump(wd + "/x.bin", x);
        res << "iterations " << it << "\n";

        // Tests::FGMRES_sap (src/tests.cpp:33-46): FGMRES with one SAP sweep as preconditioner
        spinor xsap(LevelV::Nsites[0], c_vector(LevelV::DOF[0], 0));
        FGMRES_SAP sap_solver(LV::Ntot, 2, FGMRESV::fgmres_restart_length, FGMRESV::fgmres_restarts,
                              FGMRESV::fgmres_tolerance, GConf.Conf, m0);
        const int its = sap_solver.fgmres(rhs, x0, xsap, false, false);
        dump(wd + "/x_sap.bin", xsap);
        res << "sap_solver_iterations " << its << "\n";

        // Tests::GMRES, Tests::CG, Tests::BiCG (src/tests.cpp:5-31): the comparison solvers
        spinor xg(LevelV::Nsites[0], c_vector(LevelV::DOF[0], 0));
        FGMRES_fine_level gmres(LV::Ntot, 2, 20, 50, 1e-10, GConf.Conf, m0);
        res << "gmres_iterations " << gmres.fgmres(rhs, x0, xg, false, false) << "\n";
        dump(wd + "/x_gmres.bin", xg);
        spinor xc(LevelV::Nsites[0], c_vector(LevelV::DOF[0], 0));
        res << "cg_iterations " << conjugate_gradient(GConf.Conf, rhs, xc, m0) << "\n";
        dump(wd + "/x_cg.bin", xc);
        const spinor xb = bi_cgstab(&D_phi, LV::Ntot, 2, GConf.Conf, rhs, x0, m0, 100000, 1e-10, false, false);
        dump(wd + "/x_bicg.bin", xb);

        spinor d(LevelV::Nsites[0], c_vector(2, 0));
        D_phi(GConf.Conf, rhs, d, m0);
        dump(wd + "/dphi.bin", d);
        D_dagger_phi(GConf.Conf, rhs, d, m0);
        dump(wd + "/ddagphi.bin", d);

        // the hierarchy's operations (AlgebraicMG with the same draw and set-up)
        AlgebraicMG amg(GConf, m0, AMGV::nu1, AMGV::nu2);
        amg.setUpPhase(AMGV::Nit);
        for (int l = 0; l < AMGV::levels; l++) {
            spinor pv(LevelV::Nsites[l], c_vector(LevelV::DOF[l], 0));
            if (!load(wd + "/probe_l" + std::to_string(l) + ".bin", pv)) continue;
            spinor out(LevelV::Nsites[l], c_vector(LevelV::DOF[l], 0));
            amg.levels[l]->D_operator(pv, out);
            dump(wd + "/dop_l" + std::to_string(l) + ".bin", out);
            if (l == 0) {
                spinor c(LevelV::Nsites[1], c_vector(LevelV::DOF[1], 0));
                amg.levels[0]->Pt_v(pv, c);
                dump(wd + "/pt_l0.bin", c);
                spinor pc(LevelV::Nsites[0], c_vector(LevelV::DOF[0], 0));
                amg.levels[0]->P_v(c, pc);
                dump(wd + "/ppt_l0.bin", pc);
                spinor xs(LevelV::Nsites[0], c_vector(LevelV::DOF[0], 0));
                const int ret = amg.levels[0]->sap_l.SAP(pv, xs, 2, SAPV::sap_blocks_per_proc, false);
                dump(wd + "/sap_l0.bin", xs);
                res << "sap_ret_l0 " << ret << "\n";
            }
            if (l == AMGV::levels - 1) {
                spinor xg(LevelV::Nsites[l], c_vector(LevelV::DOF[l], 0));
                const int git = amg.levels[l]->gmres_l.fgmres(pv, pv, xg, false, false);
                dump(wd + "/gmres_l" + std::to_string(l) + ".bin", xg);
                res << "gmres_iters_l" << l << " " << git << "\n";
            }
        }
        spinor z(LevelV::Nsites[0], c_vector(2, 0));
        amg.k_cycle(0, rhs, z);
        dump(wd + "/cycle0_rhs.bin", z);
        // the stand-alone multigrid solver: K-cycles to 1e-10
        spinor xm(LevelV::Nsites[0], c_vector(2, 0));
        amg.applyMultilevel(200, rhs, xm, 1e-10, true);
        spinor dxm(LevelV::Nsites[0], c_vector(2, 0));
        D_phi(GConf.Conf, xm, dxm, m0);
        double rn = 0, bn = 0;
        for (int n = 0; n < LV::Ntot; n++)
            for (int s = 0; s < 2; s++) {
                rn += std::norm(rhs[n][s] - dxm[n][s]);
                bn += std::norm(rhs[n][s]);
            }
        res << "multilevel_rel_residual " << std::sqrt(rn / bn) << "\n";
    } catch (const amg_b200::Error& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
