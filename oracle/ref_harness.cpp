/*
 * Oracle harness around the UNMODIFIED reference solver (Fabian2598/AMG_SchwingerModel).
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/build_ref.sh compiles this file together with the
 * reference's own src/*.cpp (all but src/main.cpp) into oracle/_ref/ref_<NS>x<NT>_l<LEVELS>.
 * The binary is the checker the GPU library is compared against; it is never linked
 * into, or called by, the product library.
 *
 * Usage:  ref_<NS>x<NT>_l<LEVELS> <workdir>
 *   <workdir>/params.dat   parameters.dat rows "level bx bt ntest sbx sbt" (include/params.h:17-69)
 *   <workdir>/job.txt      "key value" lines (see read_job below)
 *   <workdir>/gauge.bin    U[N][2] complex128, n = x*Nt + t (src/gauge_conf.cpp:18-32 layout)
 *   <workdir>/rhs.bin      b[N][2] complex128
 *   <workdir>/probe_l<l>.bin  optional per-level probe vectors [N_l][DOF_l] complex128
 * Outputs (raw little-endian arrays, listed with dtype and shape in <workdir>/manifest.txt).
 * With `ranks N` in job.txt the job runs as N processes (the reference's MPI layout, see
 * oracle/mpi_shim/mpi.h); rank 0 writes the outputs above, ranks r > 0 write theirs under
 * <workdir>/rank<r>/.
 *
 * The reference's private members are needed to dump the set-up hierarchy that
 * FGMRES_AMG builds in its constructor (include/amg.h:101-119); they are opened by
 * redefining `private` for the reference headers only, after every standard header
 * has been included.
 */
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <numeric>
#include <random>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include <sys/stat.h>

#define private public
#include "params.h"
#include "boundary.h"
#include "amg.h"
#include "bi_cgstab.h"
#include "conjugate_gradient.h"
#undef private

namespace {

std::string g_dir;   // the job's directory: inputs, and rank 0's outputs
std::string g_out;   // where this rank writes (rank r > 0: <workdir>/rank<r>)
std::ofstream g_manifest;

double now_s() {
    using clk = std::chrono::steady_clock;
    return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

void dump_raw(const std::string& name, const void* data, size_t bytes, const char* dtype,
              const std::vector<long>& shape) {
    std::ofstream f(g_out + "/" + name + ".bin", std::ios::binary);
    f.write(reinterpret_cast<const char*>(data), (std::streamsize)bytes);
    g_manifest << name << " " << dtype;
    for (long s : shape) g_manifest << " " << s;
    g_manifest << "\n";
}

void dump_spinor(const std::string& name, const spinor& v) {
    std::vector<c_double> flat;
    long d2 = v.empty() ? 0 : (long)v[0].size();
    flat.reserve(v.size() * d2);
    for (auto& row : v) flat.insert(flat.end(), row.begin(), row.end());
    dump_raw(name, flat.data(), flat.size() * sizeof(c_double), "c16", {(long)v.size(), d2});
}

void dump_cvec(const std::string& name, const c_vector& v) {
    dump_raw(name, v.data(), v.size() * sizeof(c_double), "c16", {(long)v.size()});
}

void dump_ivec(const std::string& name, const std::vector<int>& v) {
    dump_raw(name, v.data(), v.size() * sizeof(int), "i4", {(long)v.size()});
}

// Runs the rest of the job as `ranks` processes (oracle/mpi_shim/mpi.h), the reference's
// MPI layout on this host's cores: the SAP blocks of each colour are split among the ranks
// as SAPV::sap_blocks_per_proc says (src/sap.cpp:77-78), everything else is repeated by
// every rank.  Ranks r > 0 write under <workdir>/rank<r>/ from here on; `info`, when given,
// is flushed before the fork and reopened there by those ranks.  Started after the set-up,
// the ranks share its pages copy-on-write; an MPI run holds the same hierarchy on every rank
// (one seed for all ranks, src/amg.cpp:8, and exact SAP sums), so what follows is the
// np-rank run's.
bool start_ranks(int ranks, std::ofstream* info) {
    if (ranks <= 1) return true;
    size_t slot = 0;
    int coloring = 1;
    for (int l = 0; l < AMGV::levels; l++) {
        slot = std::max(slot, (size_t)LevelV::Nsites[l] * LevelV::DOF[l] * sizeof(c_double));
        const int nb = LevelV::SAP_Block_x[l] * LevelV::SAP_Block_t[l];
        coloring = std::max(coloring, nb != 1 ? nb / 2 : 1);
    }
    if (info) info->flush();
    if (g_manifest.is_open()) g_manifest.flush();
    std::cout.flush();
    std::cerr.flush();
    oracle_mpi_spawn(ranks, slot);
    SAPV::sap_blocks_per_proc = (coloring + ranks - 1) / ranks;
    if (oracle_mpi().rank == 0) return true;
    g_out = g_dir + "/rank" + std::to_string(oracle_mpi().rank);
    mkdir(g_out.c_str(), 0755);
    if (chdir(g_out.c_str()) != 0) {
        std::cerr << "cannot enter " << g_out << "\n";
        return false;
    }
    if (info) {
        info->close();
        info->open(g_out + "/info.txt");
        *info << std::setprecision(17);
    }
    if (g_manifest.is_open()) {
        g_manifest.close();
        g_manifest.open(g_out + "/manifest.txt");
    }
    return true;
}

bool read_spinor(const std::string& path, spinor& v) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    for (auto& row : v) f.read(reinterpret_cast<char*>(row.data()), (std::streamsize)(row.size() * sizeof(c_double)));
    return (bool)f;
}

std::map<std::string, std::string> read_job(const std::string& path) {
    std::map<std::string, std::string> kv;
    std::ifstream f(path);
    std::string k, v;
    while (f >> k >> v) kv[k] = v;
    return kv;
}

double jd(const std::map<std::string, std::string>& kv, const std::string& k, double def) {
    auto it = kv.find(k);
    return it == kv.end() ? def : std::atof(it->second.c_str());
}

// Replica of the initial test-vector draw of AlgebraicMG::setUpPhase (src/amg.cpp:8-35):
// a fresh mt19937(50) with the same uniform(-1,1) expression, so the values equal the ones
// the reference's function-local static generator produces on its first call in a process.
// Level l>=1 columns i < Ntest[l-1] are P^dagger of the (still random) level l-1 columns.
void replica_initial_test_vectors(AlgebraicMG& amg, std::vector<std::vector<spinor>>& out) {
    std::mt19937 randomInt(50);
    std::uniform_real_distribution<double> distribution(-1.0, 1.0);
    out.assign(AMGV::levels - 1, {});
    for (int l = 0; l < AMGV::levels - 1; l++)
        out[l].assign(LevelV::Ntest[l], spinor(LevelV::Nsites[l], c_vector(LevelV::DOF[l], 0)));
    for (int i = 0; i < LevelV::Ntest[0]; i++)
        for (int n = 0; n < LevelV::Nsites[0]; n++)
            for (int dof = 0; dof < LevelV::DOF[0]; dof++)
                out[0][i][n][dof] = distribution(randomInt) + I_number * distribution(randomInt);
    // Pt_v reads levels[l-1]->interpolator_columns, so stage the replica there temporarily.
    std::vector<std::vector<spinor>> saved(AMGV::levels - 1);
    for (int l = 0; l < AMGV::levels - 1; l++) saved[l] = amg.levels[l]->interpolator_columns;
    amg.levels[0]->interpolator_columns = out[0];
    for (int l = 1; l < AMGV::levels - 1; l++) {
        for (int i = 0; i < LevelV::Ntest[l]; i++) {
            if (i < LevelV::Ntest[l - 1]) {
                amg.levels[l - 1]->Pt_v(amg.levels[l - 1]->interpolator_columns[i], out[l][i]);
            } else {
                for (int n = 0; n < LevelV::Nsites[l]; n++)
                    for (int dof = 0; dof < LevelV::DOF[l]; dof++)
                        out[l][i][n][dof] = distribution(randomInt) + I_number * distribution(randomInt);
            }
        }
        amg.levels[l]->interpolator_columns = out[l];
    }
    for (int l = 0; l < AMGV::levels - 1; l++) amg.levels[l]->interpolator_columns = saved[l];
}

void dump_geometry() {
    for (int l = 0; l < AMGV::levels; l++) {
        int N = LevelV::Nsites[l];
        std::vector<int> r(N * 2), lft(N * 2), sr(N * 2), sl(N * 2);
        for (int n = 0; n < N; n++)
            for (int mu = 0; mu < 2; mu++) {
                r[2 * n + mu] = RightPB_l[l][n][mu];
                lft[2 * n + mu] = LeftPB_l[l][n][mu];
                sr[2 * n + mu] = (int)std::real(SignR_l[l][n][mu]);
                sl[2 * n + mu] = (int)std::real(SignL_l[l][n][mu]);
            }
        std::string s = std::to_string(l);
        dump_ivec("rightpb_l" + s, r);
        dump_ivec("leftpb_l" + s, lft);
        dump_ivec("signr_l" + s, sr);
        dump_ivec("signl_l" + s, sl);
    }
}

void dump_level_maps(AlgebraicMG& amg) {
    for (int l = 0; l < AMGV::levels; l++) {
        Level& L = *amg.levels[l];
        std::string s = std::to_string(l);
        if (l < AMGV::levels - 1) {
            std::vector<int> blocks;
            for (auto& b : L.LatticeBlocks) blocks.insert(blocks.end(), b.begin(), b.end());
            dump_ivec("latblocks_l" + s, blocks);
            int nagg = L.NBlocks * 2 * L.sites_per_block * L.colors;
            dump_ivec("agg_l" + s, std::vector<int>(L.Agg, L.Agg + nagg));
            int nc = L.Nsites * 2 * L.colors;
            dump_ivec("ncoords_l" + s, std::vector<int>(L.nCoords, L.nCoords + nc));
            dump_ivec("scoords_l" + s, std::vector<int>(L.sCoords, L.sCoords + nc));
            dump_ivec("ccoords_l" + s, std::vector<int>(L.cCoords, L.cCoords + nc));
        }
        std::vector<int> sblocks;
        for (auto& b : L.sap_l.Blocks) sblocks.insert(sblocks.end(), b.begin(), b.end());
        dump_ivec("sapblocks_l" + s, sblocks);
        dump_ivec("sapred_l" + s, L.sap_l.RedBlocks);
        dump_ivec("sapblack_l" + s, L.sap_l.BlackBlocks);
    }
}

void dump_hierarchy(AlgebraicMG& amg, const std::string& tag) {
    for (int l = 0; l < AMGV::levels; l++) {
        Level& L = *amg.levels[l];
        std::string s = std::to_string(l);
        if (l < AMGV::levels - 1)
            for (int i = 0; i < L.Ntest; i++)
                dump_spinor(tag + "tv_l" + s + "_" + std::to_string(i), L.interpolator_columns[i]);
        if (l > 0) {
            dump_cvec(tag + "g1_l" + s, L.G1);
            dump_cvec(tag + "g2_l" + s, L.G2);
            dump_cvec(tag + "g3_l" + s, L.G3);
        }
    }
}

// FGMRES_AMG's two overrides (include/amg.h:130-144) over an AlgebraicMG given from outside,
// so that a hierarchy loaded from files instead of built by the constructor's setUpPhase
// drives the reference's own outer FGMRES (src/fgmres.cpp:5-88) and cycles (src/amg.cpp).
class LoadedAMGFGMRES : public FGMRES {
public:
    LoadedAMGFGMRES(const int& dim1, const int& dim2, const int& m, const int& restarts, const double& tol,
                    const GaugeConf& g, double m0, AlgebraicMG& amg)
        : FGMRES(dim1, dim2, m, restarts, tol), g_(g), m0_(m0), amg_(amg) {}

private:
    const GaugeConf& g_;
    const double m0_;
    AlgebraicMG& amg_;
    void func(const spinor& in, spinor& out) override { D_phi(g_.Conf, in, out, m0_); }
    void preconditioner(const spinor& in, spinor& out) override {
        for (auto& row : out)
            for (auto& v : row) v = 0;
        if (AMGV::cycle == 0) amg_.v_cycle(0, in, out);
        else if (AMGV::cycle == 1) amg_.k_cycle(0, in, out);
    }
};

// Runs `solve` (one complete outer solve from x0 = 0, returning the reference's iteration
// count; `last` says whether to print and save the residual history) up to `reps` times, at
// least once, while rank 0's summed solve time stays below `budget` seconds (0: no budget).
// With several ranks the stop decision uses rank 0's clock on every rank (an all-reduce sum
// with zeros elsewhere), so all ranks run the same number of solves.  Writes
// solve_seconds_<r> / iterations_<r> per solve and solves_done; returns the last count.
template <class F>
int timed_solves(F&& solve, int reps, double budget, std::ofstream& info, double& t_last) {
    double total = 0;
    int iters = 0, done = 0;
    for (int r = 0; r < reps; r++) {
        bool last = r == reps - 1;
        if (!last && budget > 0) {
            // would one more solve of the last solve's length still fit the budget (rank 0's
            // projected total, the same on every rank)?
            double t0 = oracle_mpi().rank != 0 ? 0.0 : total + t_last;
            double tsum = t0;
            if (oracle_mpi().size > 1) MPI_Allreduce(&t0, &tsum, 1, MPI_DOUBLE, MPI_SUM, MPI_COMM_WORLD);
            if (r > 0 && tsum > budget) break;
        }
        const double t1 = now_s();
        iters = solve(last);
        t_last = now_s() - t1;
        total += t_last;
        done++;
        info << "solve_seconds_" << r << " " << t_last << "\n";
        info << "iterations_" << r << " " << iters << "\n";
    }
    info << "solves_done " << done << "\n";
    return iters;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::cerr << "usage: " << argv[0] << " <workdir>\n";
        return 2;
    }
    {
        char* abs = realpath(argv[1], nullptr);
        if (!abs) { std::cerr << "workdir " << argv[1] << " not found\n"; return 2; }
        g_dir = abs;
        std::free(abs);
    }
    auto job = read_job(g_dir + "/job.txt");

    readParameters(g_dir + "/params.dat");
    // `ranks` > 1: the reference's MPI layout on this host's cores, see start_ranks.  With
    // `ranks_after_setup` 1 the ranks start just before a timed loop instead of here.
    const int ranks = std::max(1, (int)jd(job, "ranks", 1));
    const bool late_ranks = (int)jd(job, "ranks_after_setup", 0) != 0;
    // with one rank every block of a colour is solved by this process (src/sap.cpp:77-78)
    SAPV::sap_blocks_per_proc = 1 << 30;
    g_out = g_dir;
    if (!late_ranks && !start_ranks(ranks, nullptr)) return 3;
    // failure drill for the stand-in's liveness checks: this rank leaves before its first
    // collective, as a crashed MPI rank would
    if (ranks > 1 && (int)jd(job, "drill_exit_rank", -1) == oracle_mpi().rank) std::_Exit(0);
    g_manifest.open(g_out + "/manifest.txt");
    Coordinates();
    boundary();

    AMGV::cycle = (int)jd(job, "cycle", 1);
    AMGV::Nit = (int)jd(job, "nit", 0);
    AMGV::SAP_test_vectors_iterations = (int)jd(job, "sap_tv_iters", 4);
    AMGV::nu1 = (int)jd(job, "nu1", 0);
    AMGV::nu2 = (int)jd(job, "nu2", 2);
    mass::m0 = jd(job, "m0", -0.1);
    const double m0 = mass::m0;
    const int N = LV::Ntot;

    GaugeConf GConf(LV::Nx, LV::Nt);
    {
        spinor g(N, c_vector(2, 0));
        if (!read_spinor(g_dir + "/gauge.bin", g)) { std::cerr << "gauge.bin missing\n"; return 3; }
        GConf.setGconf(g);
    }
    spinor rhs(N, c_vector(2, 0));
    if (!read_spinor(g_dir + "/rhs.bin", rhs)) { std::cerr << "rhs.bin missing\n"; return 3; }

    std::ofstream info(g_out + "/info.txt");
    info << std::setprecision(17);

    // D_phi / D_dagger_phi (src/dirac_operator.cpp:3-54) on the rhs.
    {
        spinor out(N, c_vector(2, 0)), outd(N, c_vector(2, 0));
        D_phi(GConf.Conf, rhs, out, m0);
        D_dagger_phi(GConf.Conf, rhs, outd, m0);
        dump_spinor("dphi", out);
        dump_spinor("ddagphi", outd);
        int reps = (int)jd(job, "dphi_reps", 0);
        if (reps > 0) {
            double t0 = now_s();
            for (int r = 0; r < reps; r++) D_phi(GConf.Conf, rhs, out, m0);
            info << "dphi_seconds_per_apply " << (now_s() - t0) / reps << "\n";
        }
    }
    // The comparison solvers (src/conjugate_gradient.cpp:5-65, src/bi_cgstab.cpp:5-89) on the
    // rhs, as Tests::CG and Tests::BiCG run them (src/tests.cpp:3-31); their iteration counts
    // are in the reference's own stdout lines.
    if ((int)jd(job, "krylov", 0)) {
        spinor y(N, c_vector(2, 0));
        conjugate_gradient(GConf.Conf, rhs, y, m0);
        dump_spinor("cg_x", y);
        const spinor x0(N, c_vector(2, 0));
        const spinor xb = bi_cgstab(&D_phi, N, 2, GConf.Conf, rhs, x0, m0, (int)jd(job, "bicg_max_iter", 100000),
                                    1e-10, true, false);
        dump_spinor("bicg_x", xb);
        // Tests::GMRES (src/tests.cpp:13-22): FGMRES_fine_level(20, 50, 1e-10), x0 = 0
        FGMRES_fine_level fg(N, 2, 20, 50, 1e-10, GConf.Conf, m0);
        spinor xg(N, c_vector(2, 0));
        const int git = fg.fgmres(rhs, x0, xg, false, false);
        dump_spinor("gmres_x", xg);
        info << "gmres_iterations " << git << "\n";
        // Tests::FGMRES_sap (src/tests.cpp:33-46) with the global SAP object given the gauge
        // field first through its public SAP_fine_level::set_params (include/sap.h:145-148),
        // which the reference's own main never calls: FGMRES(20, 50, 1e-10) with one SAP
        // sweep on SAPV::sap_block_x x sap_block_t blocks as preconditioner
        sap.set_params(GConf.Conf, m0);
        FGMRES_SAP fs(N, 2, 20, 50, 1e-10, GConf.Conf, m0);
        spinor xs(N, c_vector(2, 0));
        const int sit = fs.fgmres(rhs, x0, xs, false, false);
        dump_spinor("sap_x", xs);
        info << "sap_iterations " << sit << "\n";
        std::cout.flush();
        g_manifest.close();
        return 0;
    }
    if ((int)jd(job, "dphi_only", 0)) { g_manifest.close(); return 0; }

    dump_geometry();

    if ((int)jd(job, "phases", 0)) {
        // A stand-alone hierarchy (same constructor as FGMRES_AMG uses) for maps and the
        // initial test-vector replica; set-up is not run on it, so the static RNG of
        // setUpPhase is untouched for the FGMRES_AMG solve below.
        AlgebraicMG probe(GConf, m0, AMGV::nu1, AMGV::nu2);
        dump_level_maps(probe);
        std::vector<std::vector<spinor>> tv0;
        replica_initial_test_vectors(probe, tv0);
        for (int l = 0; l < AMGV::levels - 1; l++)
            for (int i = 0; i < LevelV::Ntest[l]; i++)
                dump_spinor("init_tv_l" + std::to_string(l) + "_" + std::to_string(i), tv0[l][i]);
    }

    if (!(int)jd(job, "solve", 1)) { g_manifest.close(); return 0; }

    // Bounded CPU sample on a given hierarchy: the reference's AlgebraicMG is constructed
    // without its set-up, the test vectors and coarse links are loaded from
    // hier_tv_l<l>.bin / hier_g{1,2,3}_l<l>.bin, and one outer iteration (the preconditioner
    // of FGMRES_AMG::preconditioner, include/amg.h:134-144, plus D_phi) is timed.
    if ((int)jd(job, "load_hierarchy", 0)) {
        AlgebraicMG amgh(GConf, m0, AMGV::nu1, AMGV::nu2);
        for (int l = 0; l < AMGV::levels; l++) {
            Level& L = *amgh.levels[l];
            std::string sl = std::to_string(l);
            if (l < AMGV::levels - 1) {
                std::ifstream f(g_dir + "/hier_tv_l" + sl + ".bin", std::ios::binary);
                if (!f) { std::cerr << "missing hierarchy test vectors l" << l << "\n"; return 3; }
                for (auto& v : L.interpolator_columns)
                    for (auto& row : v) f.read(reinterpret_cast<char*>(row.data()), (std::streamsize)(row.size() * sizeof(c_double)));
            }
            if (l > 0) {
                for (auto pr : {std::make_pair("g1", &L.G1), std::make_pair("g2", &L.G2), std::make_pair("g3", &L.G3)}) {
                    std::ifstream f(g_dir + "/hier_" + pr.first + "_l" + sl + ".bin", std::ios::binary);
                    if (!f) { std::cerr << "missing hierarchy links l" << l << "\n"; return 3; }
                    f.read(reinterpret_cast<char*>(pr.second->data()), (std::streamsize)(pr.second->size() * sizeof(c_double)));
                }
            }
        }
        if ((int)jd(job, "solve_reps", 0) > 0) {
            // complete outer solves (FGMRES_AMG::fgmres, x0 = 0) on the loaded hierarchy
            static const int dim1 = LV::Ntot, dim2 = 2;
            LoadedAMGFGMRES fs(dim1, dim2, FGMRESV::fgmres_restart_length, FGMRESV::fgmres_restarts,
                               FGMRESV::fgmres_tolerance, GConf, m0, amgh);
            spinor x0(N, c_vector(2, 0)), x(N, c_vector(2, 0));
            if (late_ranks && !start_ranks(ranks, &info)) return 3;
            double t_last = 0;
            const int iters = timed_solves([&](bool last) { return fs.fgmres(rhs, x0, x, last, last); },
                                           (int)jd(job, "solve_reps", 1), jd(job, "solve_budget_seconds", 0), info,
                                           t_last);
            dump_spinor("x", x);
            spinor Dx(N, c_vector(2, 0));
            D_phi(GConf.Conf, x, Dx, m0);
            double rr = 0, bb = 0;
            for (int n = 0; n < N; n++)
                for (int a = 0; a < 2; a++) {
                    rr += std::norm(rhs[n][a] - Dx[n][a]);
                    bb += std::norm(rhs[n][a]);
                }
            info << "true_rel_residual " << std::sqrt(rr / bb) << "\n";
            info << "iterations " << iters << "\n";
            info << "solve_seconds " << t_last << "\n";
            g_manifest.close();
            return 0;
        }
        const int reps = std::max(1, (int)jd(job, "outer_iteration_reps", 1));
        spinor v(N, c_vector(2, 0)), z(N, c_vector(2, 0)), w(N, c_vector(2, 0));
        double nb = std::sqrt(std::real(dot(rhs, rhs)));
        for (int n = 0; n < N; n++) for (int a = 0; a < 2; a++) v[n][a] = rhs[n][a] / nb;
        if (late_ranks && !start_ranks(ranks, &info)) return 3;
        for (int r = 0; r < reps; r++) {
            double t1 = now_s();
            for (auto& row : z) { row[0] = 0; row[1] = 0; }
            if (AMGV::cycle == 1) amgh.k_cycle(0, v, z); else amgh.v_cycle(0, v, z);
            D_phi(GConf.Conf, z, w, m0);
            info << "outer_iteration_seconds_" << r << " " << (now_s() - t1) << "\n";
        }
        dump_spinor("sample_z", z);
        g_manifest.close();
        return 0;
    }

    spinor x0(N, c_vector(2, 0)), x(N, c_vector(2, 0));
    // FGMRES_AMG keeps its dim1/dim2 arguments by reference (include/amg.h:125-126), so they
    // must outlive the object; src/tests.cpp:72 passes the literal 2, a dangling reference.
    static const int dim1 = LV::Ntot, dim2 = 2;
    double t0 = now_s();
    FGMRES_AMG f_amg(dim1, dim2, FGMRESV::fgmres_restart_length, FGMRESV::fgmres_restarts,
                     FGMRESV::fgmres_tolerance, GConf, m0);
    double t_setup = now_s() - t0;
    AlgebraicMG& amg = f_amg.amg;
    if ((int)jd(job, "dump_hierarchy", 1)) dump_hierarchy(amg, "");

    if ((int)jd(job, "phases", 0)) {
        // Per-level operator probes on the set-up hierarchy.
        for (int l = 0; l < AMGV::levels; l++) {
            std::string s = std::to_string(l);
            spinor pv(LevelV::Nsites[l], c_vector(LevelV::DOF[l], 0));
            if (!read_spinor(g_dir + "/probe_l" + s + ".bin", pv)) continue;
            spinor out(LevelV::Nsites[l], c_vector(LevelV::DOF[l], 0));
            amg.levels[l]->D_operator(pv, out);
            dump_spinor("dop_l" + s, out);
            if (l < AMGV::levels - 1) {
                spinor c(LevelV::Nsites[l + 1], c_vector(LevelV::DOF[l + 1], 0));
                amg.levels[l]->Pt_v(pv, c);
                dump_spinor("pt_l" + s, c);
                spinor pc(LevelV::Nsites[l], c_vector(LevelV::DOF[l], 0));
                amg.levels[l]->P_v(c, pc);
                dump_spinor("ppt_l" + s, pc);
                // One SAP call (src/sap.cpp:64-174): D x = probe from x = 0 and from x = probe.
                spinor xs(LevelV::Nsites[l], c_vector(LevelV::DOF[l], 0));
                int ret = amg.levels[l]->sap_l.SAP(pv, xs, (int)jd(job, "sap_probe_nu", 2), SAPV::sap_blocks_per_proc, false);
                dump_spinor("sap_l" + s, xs);
                info << "sap_ret_l" << s << " " << ret << "\n";
            }
            // One level-l GMRES of the kind the cycles use at the coarsest level
            // (include/level.h:66-85), x0 = rhs as in src/amg.cpp:138.
            if (l == 0) continue;
            spinor xg(LevelV::Nsites[l], c_vector(LevelV::DOF[l], 0));
            int it = amg.levels[l]->gmres_l.fgmres(pv, pv, xg, false, false);
            dump_spinor("gmres_l" + s, xg);
            info << "gmres_iters_l" << s << " " << it << "\n";
        }
        // One preconditioner application from the fine level (src/amg.cpp:135-178 / :90-132).
        {
            spinor z(N, c_vector(2, 0));
            if (AMGV::cycle == 1) amg.k_cycle(0, rhs, z); else amg.v_cycle(0, rhs, z);
            dump_spinor("cycle0_rhs", z);
        }
        if (AMGV::levels > 2) {
            spinor pv(LevelV::Nsites[1], c_vector(LevelV::DOF[1], 0));
            if (read_spinor(g_dir + "/probe_l1.bin", pv)) {
                spinor z(LevelV::Nsites[1], c_vector(LevelV::DOF[1], 0));
                if (AMGV::cycle == 1) amg.k_cycle(1, pv, z); else amg.v_cycle(1, pv, z);
                dump_spinor("cycle1_probe", z);
                spinor z2(LevelV::Nsites[1], c_vector(LevelV::DOF[1], 0));
                int it = amg.fgmres_k_cycle_l[1]->fgmres(pv, pv, z2, false, false);
                dump_spinor("kfgmres1_probe", z2);
                info << "kfgmres1_iters " << it << "\n";
            }
        }
    }

    // Bounded CPU sample: one outer FGMRES iteration of the reference -- the preconditioner
    // application (FGMRES_AMG::preconditioner: zero, then one cycle from level 0) plus the
    // D_phi of the Arnoldi step -- timed `outer_iteration_reps` times.
    if ((int)jd(job, "outer_iteration_reps", 0) > 0) {
        const int reps = (int)jd(job, "outer_iteration_reps", 0);
        spinor v(N, c_vector(2, 0)), z(N, c_vector(2, 0)), w(N, c_vector(2, 0));
        double nb = std::sqrt(std::real(dot(rhs, rhs)));
        for (int n = 0; n < N; n++) for (int a = 0; a < 2; a++) v[n][a] = rhs[n][a] / nb;
        if (late_ranks && !start_ranks(ranks, &info)) return 3;
        double t1 = now_s();
        for (int r = 0; r < reps; r++) {
            double t2 = now_s();
            for (auto& row : z) { row[0] = 0; row[1] = 0; }
            if (AMGV::cycle == 1) amg.k_cycle(0, v, z); else amg.v_cycle(0, v, z);
            D_phi(GConf.Conf, z, w, m0);
            info << "outer_iteration_seconds_" << r << " " << (now_s() - t2) << "\n";
        }
        info << "outer_iteration_seconds " << (now_s() - t1) / reps << "\n";
        info << "setup_seconds " << t_setup << "\n";
        dump_spinor("sample_z", z);
        g_manifest.close();
        return 0;
    }

    // The outer solve (src/tests.cpp:67-82): FGMRES_AMG::fgmres(rhs, x0 = 0, x).  With
    // `solve_reps` R > 1 the complete solve is repeated up to R times on the same hierarchy
    // (each call starts from x0 = 0 and re-zeroes the solver's state, src/fgmres.cpp:6-9),
    // each one timed, within `solve_budget_seconds`; the ranks of `ranks_after_setup` start
    // just before the first.
    const int solve_reps = std::max(1, (int)jd(job, "solve_reps", 1));
    if (late_ranks && !start_ranks(ranks, &info)) return 3;
    double t_solve = 0;
    const int iters = timed_solves([&](bool last) { return f_amg.fgmres(rhs, x0, x, last, last); }, solve_reps,
                                   jd(job, "solve_budget_seconds", 0), info, t_solve);
    dump_spinor("x", x);
    {
        spinor Dx(N, c_vector(2, 0));
        D_phi(GConf.Conf, x, Dx, m0);
        double rr = 0, bb = 0;
        for (int n = 0; n < N; n++)
            for (int a = 0; a < 2; a++) {
                rr += std::norm(rhs[n][a] - Dx[n][a]);
                bb += std::norm(rhs[n][a]);
            }
        info << "true_rel_residual " << std::sqrt(rr / bb) << "\n";
    }
    info << "iterations " << iters << "\n";
    info << "setup_seconds " << t_setup << "\n";
    info << "solve_seconds " << t_solve << "\n";
    g_manifest.close();
    return 0;
}
