/*
 * amg_b200.hpp -- C++ classes with the reference's names and signatures
 * (Fabian2598/AMG_SchwingerModel) over the C ABI of libschwinger_amg.so.
 *
 * A program written against the reference's headers builds against this one instead:
 * define NS, NT and LEVELS (what the reference's CMake writes into config.h,
 * include/config.h.in:3-5), include this header in place of variables.h / params.h /
 * gauge_conf.h / dirac_operator.h / fgmres.h / level.h / amg.h, and link
 * -lschwinger_amg.  The solver runs on the GPU; the classes keep the reference's host
 * types (spinor = vector<vector<complex<double>>>) and copy at the boundary.
 *
 * Differences from the reference, all at the error path: a missing file or a failed call
 * throws amg_b200::Error (the reference prints and calls exit(1)); nothing here uses MPI.
 */
#ifndef AMG_B200_HPP
#define AMG_B200_HPP

#if !defined(NS) || !defined(NT) || !defined(LEVELS)
#error "define NS, NT and LEVELS (the lattice size and level count) before including amg_b200.hpp"
#endif

#include <cmath>
#include <complex>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../schwinger_amg.h"

// ---- types (include/lin_alg_op.h:11-14, include/variables.h:11) ------------------------
typedef std::complex<double> c_double;
typedef std::vector<c_double> c_vector;
typedef std::vector<c_vector> c_matrix;
typedef std::vector<c_vector> spinor;

// ---- lattice and solver parameters (include/variables.h:24-118) -----------------------
// Defaults are the reference's (src/variables.cpp:46-87); user code sets them as it would
// set the reference's globals.
namespace LV {
constexpr int Nx = NS;
constexpr int Nt = NT;
constexpr int Ntot = Nx * Nt;
}  // namespace LV

namespace SAPV {
inline int sap_gmres_restart_length = 5;
inline int sap_gmres_restarts = 5;
inline double sap_gmres_tolerance = 1e-3;
inline double sap_tolerance = 1e-10;
inline int sap_blocks_per_proc = 1;  // accepted and ignored: every block is solved on the GPU
// blocks per direction of the fine SAP that FGMRES_SAP uses (include/variables.h:35-36)
constexpr int sap_block_x = 4;
constexpr int sap_block_t = 4;
}  // namespace SAPV

namespace AMGV {
constexpr int levels = LEVELS;
inline int SAP_test_vectors_iterations = 2;
inline int gmres_restarts_coarse_level = 10;
inline int gmres_restart_length_coarse_level = 20;
inline double gmres_tol_coarse_level = 0.1;
inline int gmres_restarts_smoother = 20;
inline int nu1 = 0;
inline int nu2 = 2;
inline int Nit = 1;
inline bool SetUpDone = false;
inline int fgmres_k_cycle_restart_length = 5;
inline int fgmres_k_cycle_restarts = 2;
inline double fgmres_k_cycle_tol = 0.1;
inline int cycle = 0;
}  // namespace AMGV

namespace FGMRESV {
inline double fgmres_tolerance = 1e-10;
inline int fgmres_restart_length = 20;
inline int fgmres_restarts = 50;
}  // namespace FGMRESV

namespace CG {
inline int max_iter = 100000;
inline double tol = 1e-10;
}  // namespace CG

namespace LevelV {
constexpr int maxLevel = AMGV::levels - 1;
inline int BlocksX[AMGV::levels - 1] = {};
inline int BlocksT[AMGV::levels - 1] = {};
inline int Ntest[AMGV::levels - 1] = {};
inline int Nagg[AMGV::levels - 1] = {};
inline int NBlocks[AMGV::levels - 1] = {};
inline int Nsites[AMGV::levels] = {};
inline int NxSites[AMGV::levels] = {};
inline int NtSites[AMGV::levels] = {};
inline int DOF[AMGV::levels] = {};
inline int Colors[AMGV::levels] = {};
inline int SAP_Block_x[AMGV::levels] = {};
inline int SAP_Block_t[AMGV::levels] = {};
inline int GMRES_restart_len[AMGV::levels] = {};
inline int GMRES_restarts[AMGV::levels] = {};
inline double GMRES_tol[AMGV::levels] = {};
inline int SAP_elements_x[AMGV::levels] = {};
inline int SAP_elements_t[AMGV::levels] = {};
inline int SAP_variables_per_block[AMGV::levels] = {};
}  // namespace LevelV

// bare mass of the reference's main and reports (include/variables.h:20-22)
namespace mass {
inline double m0 = 0;
}  // namespace mass

namespace amg_b200 {

struct Error : std::runtime_error {
    int status;
    Error(int st, const std::string& where)
        : std::runtime_error(where + ": " + amg_status_string(st) + " (" + amg_last_error() + ")"), status(st) {}
};

inline int check(int st, const char* where) {
    if (st < 0) throw Error(st, where);
    return st;
}

// spinor [n][dof] <-> contiguous interleaved complex128
inline std::vector<c_double> flatten(const spinor& s) {
    std::vector<c_double> f;
    f.reserve(s.empty() ? 0 : s.size() * s[0].size());
    for (const auto& row : s) f.insert(f.end(), row.begin(), row.end());
    return f;
}
inline void unflatten(const std::vector<c_double>& f, spinor& s) {
    size_t k = 0;
    for (auto& row : s)
        for (auto& v : row) v = f[k++];
}
inline const double* dptr(const std::vector<c_double>& v) { return reinterpret_cast<const double*>(v.data()); }
inline double* dptr(std::vector<c_double>& v) { return reinterpret_cast<double*>(v.data()); }

// the parameters.dat rows in the form amg_create takes, from LevelV (filled by readParameters)
inline std::vector<int> rows_from_levelv() {
    std::vector<int> rows;
    for (int l = 0; l < LevelV::maxLevel; l++) {
        if (LevelV::BlocksX[l] <= 0 || LevelV::BlocksT[l] <= 0)
            throw Error(AMG_ERR_STATE, "readParameters must run before the solver is built");
        rows.insert(rows.end(), {l, LevelV::BlocksX[l], LevelV::BlocksT[l], LevelV::Ntest[l], LevelV::SAP_Block_x[l],
                                 LevelV::SAP_Block_t[l]});
    }
    return rows;
}

// amg_params from the reference's globals
inline amg_params params_from_globals(int nit) {
    amg_params p;
    amg_params_default(&p);
    p.cycle = AMGV::cycle == 0 ? AMG_CYCLE_V : AMG_CYCLE_K;
    p.nu1 = AMGV::nu1;
    p.nu2 = AMGV::nu2;
    p.nit = nit;
    p.sap_tv_iters = AMGV::SAP_test_vectors_iterations;
    p.sap_gmres_m = SAPV::sap_gmres_restart_length;
    p.sap_gmres_restarts = SAPV::sap_gmres_restarts;
    p.sap_gmres_tol = SAPV::sap_gmres_tolerance;
    p.sap_tol = SAPV::sap_tolerance;
    p.kcycle_m = AMGV::fgmres_k_cycle_restart_length;
    p.kcycle_restarts = AMGV::fgmres_k_cycle_restarts;
    p.kcycle_tol = AMGV::fgmres_k_cycle_tol;
    if (LevelV::GMRES_restart_len[LevelV::maxLevel] > 0) {
        p.coarse_m = LevelV::GMRES_restart_len[LevelV::maxLevel];
        p.coarse_restarts = LevelV::GMRES_restarts[LevelV::maxLevel];
        p.coarse_tol = LevelV::GMRES_tol[LevelV::maxLevel];
    }
    p.outer_m = FGMRESV::fgmres_restart_length;
    p.outer_restarts = FGMRESV::fgmres_restarts;
    p.outer_tol = FGMRESV::fgmres_tolerance;
    p.precision = AMG_PREC_F64;
    return p;
}

// One solver context (device memory, stream, hierarchy), created from the globals.
class Context {
public:
    Context(const c_matrix& U, double m0, int nit, int precision = AMG_PREC_F64) : nit_(nit) {
        std::vector<int> rows = rows_from_levelv();
        amg_params p = params_from_globals(nit);
        p.precision = precision;
        check(amg_create(&ctx_, LV::Nx, LV::Nt, AMGV::levels, rows.data(), m0, &p, 0), "amg_create");
        std::vector<c_double> u = flatten(U);
        check(amg_set_gauge(ctx_, dptr(u)), "amg_set_gauge");
    }
    ~Context() {
        if (ctx_) amg_destroy(ctx_);
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    amg_ctx get() const { return ctx_; }
    int nit() const { return nit_; }

private:
    amg_ctx ctx_ = nullptr;
    int nit_ = 0;
};

}  // namespace amg_b200

// ---- readParameters (include/params.h:17-69) -----------------------------------------
inline void readParameters(const std::string& inputFile) {
    int rows[6 * 16];
    int n = 0;
    amg_b200::check(amg_read_parameters(inputFile.c_str(), rows, 16, &n), "readParameters");
    const int maxLevel = LevelV::maxLevel;
    for (int i = 0; i < n; i++) {
        const int* r = rows + 6 * i;
        const int level = r[0];
        if (level < 0 || level >= maxLevel) continue;
        LevelV::BlocksX[level] = r[1];
        LevelV::BlocksT[level] = r[2];
        LevelV::Ntest[level] = r[3];
        LevelV::Nagg[level] = 2 * r[1] * r[2];
        LevelV::NBlocks[level] = r[1] * r[2];
        LevelV::SAP_Block_x[level] = r[4];
        LevelV::SAP_Block_t[level] = r[5];
        LevelV::GMRES_restart_len[level] = 20;
        LevelV::GMRES_restarts[level] = 20;
        LevelV::GMRES_tol[level] = 1e-10;
    }
    for (int l = 0; l <= maxLevel; l++) {
        LevelV::Nsites[l] = l == 0 ? LV::Ntot : LevelV::BlocksX[l - 1] * LevelV::BlocksT[l - 1];
        LevelV::NxSites[l] = l == 0 ? LV::Nx : LevelV::BlocksX[l - 1];
        LevelV::NtSites[l] = l == 0 ? LV::Nt : LevelV::BlocksT[l - 1];
        LevelV::DOF[l] = l == 0 ? 2 : 2 * LevelV::Ntest[l - 1];
        LevelV::Colors[l] = l == 0 ? 1 : LevelV::Ntest[l - 1];
        if (l < maxLevel && LevelV::SAP_Block_x[l] > 0 && LevelV::SAP_Block_t[l] > 0) {
            LevelV::SAP_elements_x[l] = LevelV::NxSites[l] / LevelV::SAP_Block_x[l];
            LevelV::SAP_elements_t[l] = LevelV::NtSites[l] / LevelV::SAP_Block_t[l];
            LevelV::SAP_variables_per_block[l] = LevelV::DOF[l] * LevelV::SAP_elements_x[l] * LevelV::SAP_elements_t[l];
        }
    }
    LevelV::SAP_Block_x[maxLevel] = 1;
    LevelV::SAP_Block_t[maxLevel] = 1;
    LevelV::GMRES_restart_len[maxLevel] = 20;
    LevelV::GMRES_restarts[maxLevel] = 20;
    LevelV::GMRES_tol[maxLevel] = 0.1;
    std::cout << "Parameters read from " << inputFile << std::endl;
}

// ---- GaugeConf (include/gauge_conf.h:12-49) -------------------------------------------
class GaugeConf {
public:
    GaugeConf(const int& Nspace, const int& Ntime) : Nx(Nspace), Nt(Ntime), Ntot(Nspace * Ntime) {
        Conf = c_matrix(Ntot, c_vector(2, 0));
    }
    GaugeConf(const GaugeConf& o) : Conf(o.Conf), Nx(o.Nx), Nt(o.Nt), Ntot(o.Ntot) {}
    void setGconf(const c_matrix& CONF) { Conf = CONF; }
    int getNx() const { return Nx; }
    int getNt() const { return Nt; }
    // text rows "x t mu re im" (src/gauge_conf.cpp:18-32)
    void read_conf(const std::string& name) {
        std::ifstream in(name);
        if (!in) throw amg_b200::Error(AMG_ERR_INVALID, "read_conf: file " + name + " not found");
        int x, t, mu;
        double re, im;
        while (in >> x >> t >> mu >> re >> im) Conf[x * Nt + t][mu] = c_double(re, im);
        std::cout << "Conf read from " << name << std::endl;
    }
    c_matrix Conf;  // Conf[Nx*Nt][2]

private:
    int Nx, Nt, Ntot;
};

// text rows "x t spin re im" (src/variables.cpp:117-130)
inline void read_rhs(spinor& vec, const std::string& name) {
    std::ifstream in(name);
    if (!in) throw amg_b200::Error(AMG_ERR_INVALID, "read_rhs: file " + name + " not found");
    int x, t, mu;
    double re, im;
    while (in >> x >> t >> mu >> re >> im) vec[x * LV::Nt + t][mu] = c_double(re, im);
}

// ---- text output and the experiment reports (src/variables.cpp:101-155, :158-290) --------
// The file names and column layouts are the reference's, so its plotting scripts read them.

// "index  value" rows, 17 significant digits (src/variables.cpp:101-115)
inline void save_vec(const std::vector<double>& vec, const std::string& name) {
    std::ofstream f(name);
    if (!f) throw amg_b200::Error(AMG_ERR_INVALID, "save_vec: cannot open " + name);
    for (size_t n = 0; n < vec.size(); n++)
        f << n << std::setw(30) << std::setprecision(17) << std::scientific << vec[n] << "\n";
}

// "x t spin re im" rows, the format read_rhs reads (src/variables.cpp:132-155)
inline void save_rhs(const spinor& rhs, const std::string& name) {
    std::ofstream f(name);
    if (!f) throw amg_b200::Error(AMG_ERR_INVALID, "save_rhs: cannot open " + name);
    for (int n = 0; n < LV::Ntot; n++)
        for (int spin = 0; spin < 2; spin++)
            f << n / LV::Nt << std::setw(30) << n % LV::Nt << std::setw(30) << spin << std::setw(30)
              << std::setprecision(17) << std::scientific << std::real(rhs[n][spin]) << std::setw(30)
              << std::setprecision(17) << std::scientific << std::imag(rhs[n][spin]) << "\n";
}

// uniform(-1, 1) complex entries from one generator seeded on the first call, as the
// reference's function-local static std::mt19937 (src/variables.cpp:158-168); the same
// expression, so the same compiler draws the parts in the same order.
inline void random_rhs(spinor& vec, const int seed) {
    static std::mt19937 gen(seed);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    const c_double I(0, 1);
    for (int i = 0; i < LV::Ntot; i++) {
        vec[i][0] = u(gen) + I * u(gen);
        vec[i][1] = u(gen) + I * u(gen);
    }
}

// the run banner (src/variables.cpp:170-222)
inline void printParameters() {
    using std::cout;
    const char* rule = "---------------------------------------------------------------------------------------";
    cout << "******************* AMG for the Dirac matrix in the Schwinger model *******************\n";
    cout << "| Nx = " << LV::Nx << " Nt = " << LV::Nt << "\n";
    cout << "| Lattice dimension = " << LV::Ntot << "\n";
    cout << "| Number of entries of the Dirac matrix = (" << 2 * LV::Ntot << ")^2\n";
    cout << "| Bare mass parameter m0 = " << mass::m0 << "\n" << rule << "\n";
    cout << "* Blocks, aggregates and test vectors at each level\n";
    for (int l = 0; l < AMGV::levels - 1; l++)
        cout << "| Level " << l << " Block X " << LevelV::BlocksX[l] << " Block T " << LevelV::BlocksT[l]
             << " Ntest " << LevelV::Ntest[l] << " Nagg " << LevelV::Nagg[l] << " Number of lattice blocks "
             << LevelV::NBlocks[l] << " Schwarz Block T " << LevelV::SAP_Block_t[l] << " Schwarz Block X "
             << LevelV::SAP_Block_x[l] << "\n";
    cout << rule << "\n* SAP blocks\n";
    for (int l = 0; l < AMGV::levels - 1; l++)
        cout << "| Level " << l << " Schwarz Block T " << LevelV::SAP_Block_t[l] << " Schwarz Block X "
             << LevelV::SAP_Block_x[l] << " Number of blocks " << LevelV::SAP_Block_t[l] * LevelV::SAP_Block_x[l]
             << " Each block has " << LevelV::SAP_variables_per_block[l] << " variables\n";
    cout << rule << "\n* Sites and degrees of freedom at each level\n";
    for (int l = 0; l < AMGV::levels; l++)
        cout << "| Level " << l << " Nsites " << LevelV::Nsites[l] << " Nxsites " << LevelV::NxSites[l]
             << " NtSites " << LevelV::NtSites[l] << " DOF " << LevelV::DOF[l] << " Colors " << LevelV::Colors[l]
             << "\n";
    cout << rule << "\n";
    cout << "| GMRES restart length for SAP blocks = " << SAPV::sap_gmres_restart_length << "\n";
    cout << "| GMRES restarts for SAP blocks = " << SAPV::sap_gmres_restarts << "\n";
    cout << "| GMRES tolerance for SAP blocks = " << SAPV::sap_gmres_tolerance << "\n" << rule << "\n";
    cout << "* AMG parameters\n";
    if (AMGV::cycle == 0) cout << "| Cycle = V-cycle\n";
    else if (AMGV::cycle == 1) cout << "| Cycle = K-cycle\n";
    cout << "| Number of levels = " << AMGV::levels << "\n";
    cout << "| nu1 (pre-smoothing) = " << AMGV::nu1 << " nu2 (post-smoothing) = " << AMGV::nu2 << "\n";
    cout << "| Number of iterations for improving the interpolator = " << AMGV::Nit << "\n";
    cout << "| Restart length of GMRES at the coarse level = " << LevelV::GMRES_restart_len[LevelV::maxLevel] << "\n";
    cout << "| Restarts of GMRES at the coarse level = " << LevelV::GMRES_restarts[LevelV::maxLevel] << "\n";
    cout << "| GMRES tolerance for the coarse level solution = " << LevelV::GMRES_tol[LevelV::maxLevel] << "\n";
    cout << "* FGMRES with AMG preconditioning parameters\n";
    cout << "| FGMRES restart length = " << FGMRESV::fgmres_restart_length << "\n";
    cout << "| FGMRES restarts = " << FGMRESV::fgmres_restarts << "\n";
    cout << "| FGMRES tolerance = " << FGMRESV::fgmres_tolerance << "\n";
    cout << "*****************************************************************************************************"
         << std::endl;
}

// The experiment reports of the reference's main (src/variables.cpp:226-290):
// metadata_<Nx>x<Nt>_Levels<L>_{V,K}cycle.dat (the blocking rows and solver parameters, and
// the configuration id) and results_<Nx>x<Nt>_Levels<L>_{V,K}cycle.out (one row per bootstrap
// setting 2i: mean and spread of the iteration count and of the solve time over nMeas).
inline void saveParameters(double* Iter, double* dIter, double* exTime, double* dexTime, const int nMeas,
                           const int nconf) {
    std::ostringstream tag;
    tag << LV::Nx << "x" << LV::Nt << "_Levels" << AMGV::levels << (AMGV::cycle == 0 ? "_Vcycle" : "_Kcycle");
    {
        std::ofstream m("metadata_" + tag.str() + ".dat");
        if (!m) throw amg_b200::Error(AMG_ERR_INVALID, "saveParameters: cannot open metadata_" + tag.str() + ".dat");
        m << "#level, blocks_x, blocks_t, Ntest, SAP_blocks_x, SAP_blocks_t\n";
        for (int l = 0; l < AMGV::levels - 1; l++)
            m << l << std::setw(5) << LevelV::BlocksX[l] << std::setw(5) << LevelV::BlocksT[l] << std::setw(5)
              << LevelV::Ntest[l] << std::setw(5) << LevelV::SAP_Block_x[l] << std::setw(5) << LevelV::SAP_Block_t[l]
              << "\n";
        m << "#SAP_test_vectors_iterations\n" << AMGV::SAP_test_vectors_iterations << "\n";
        m << "#cycle (0 = V, 1 = K)\n" << AMGV::cycle << "\n";
        m << "#Pre-smoothing nu1, Post-smoothing nu2\n" << AMGV::nu1 << std::setw(5) << AMGV::nu2 << "\n";
        m << "#sap gmres restart length, sap gmres restarts, sap gmres tolerance\n";
        m << SAPV::sap_gmres_restart_length << std::setw(5) << SAPV::sap_gmres_restarts << std::setw(15)
          << std::scientific << std::setprecision(7) << SAPV::sap_gmres_tolerance << "\n";
        m << "#GMRES restart length coarse level, GMRES restarts coarse level, GMRES tolerance coarse level\n";
        m << LevelV::GMRES_restart_len[LevelV::maxLevel] << std::setw(5) << LevelV::GMRES_restarts[LevelV::maxLevel]
          << std::setw(15) << std::scientific << std::setprecision(7) << LevelV::GMRES_tol[LevelV::maxLevel] << "\n";
        m << "#FGMRES restart length, FGMRES restarts, FGMRES tolerance\n";
        m << FGMRESV::fgmres_restart_length << std::setw(5) << FGMRESV::fgmres_restarts << std::setw(15)
          << std::scientific << std::setprecision(7) << FGMRESV::fgmres_tolerance << "\n";
        m << "#Configuration ID analyzed: \n" << nconf << "\n";
    }
    std::ofstream r("results_" + tag.str() + ".out");
    if (!r) throw amg_b200::Error(AMG_ERR_INVALID, "saveParameters: cannot open results_" + tag.str() + ".out");
    r << "#Nit  Iterations  dIterations  exTime  dexTime\n";
    for (int i = 0; i < nMeas; i++)
        r << 2 * i << std::setw(15) << std::scientific << std::setprecision(7) << Iter[i] << std::setw(15)
          << std::scientific << std::setprecision(7) << dIter[i] << std::setw(15) << std::scientific
          << std::setprecision(7) << exTime[i] << std::setw(15) << std::scientific << std::setprecision(7)
          << dexTime[i] << "\n";
}

// ---- D_phi / D_dagger_phi (include/dirac_operator.h:14-23) ----------------------------
inline void D_phi(const c_matrix& U, const spinor& phi, spinor& out, const double& m0) {
    std::vector<c_double> u = amg_b200::flatten(U), in = amg_b200::flatten(phi), o(in.size());
    amg_b200::check(amg_dirac_apply_host(amg_b200::dptr(u), amg_b200::dptr(in), amg_b200::dptr(o), LV::Nx, LV::Nt, 1,
                                         m0, 0),
                    "D_phi");
    amg_b200::unflatten(o, out);
}
inline void D_dagger_phi(const c_matrix& U, const spinor& phi, spinor& out, const double& m0) {
    std::vector<c_double> u = amg_b200::flatten(U), in = amg_b200::flatten(phi), o(in.size());
    amg_b200::check(amg_dirac_apply_host(amg_b200::dptr(u), amg_b200::dptr(in), amg_b200::dptr(o), LV::Nx, LV::Nt, 1,
                                         m0, 1),
                    "D_dagger_phi");
    amg_b200::unflatten(o, out);
}

// ---- Level (include/level.h:14-265): the operations of one level of a set-up hierarchy -
class Level {
public:
    // SAP_C::SAP (include/sap.h:91): returns 1 if converged, 0 otherwise
    class SAP_level_l {
    public:
        explicit SAP_level_l(Level* parent) : parent(parent) {}
        int SAP(const spinor& v, spinor& x, const int& nu, const int& /*blocks_per_proc*/, const bool& print) {
            std::vector<c_double> vf = amg_b200::flatten(v), xf = amg_b200::flatten(x);
            const int st = amg_b200::check(
                amg_sap(parent->ctx(), parent->level, amg_b200::dptr(vf), amg_b200::dptr(xf), nu), "SAP");
            amg_b200::unflatten(xf, x);
            if (print) std::cout << (st == AMG_OK ? "SAP converged" : "SAP did not converge") << std::endl;
            return st == AMG_OK ? 1 : 0;
        }

    private:
        Level* parent;
    };
    // Level::GMRES_level_l (include/level.h:66-85): x = GMRES(b) with x0 = b
    class GMRES_level_l {
    public:
        explicit GMRES_level_l(Level* parent) : parent(parent) {}
        int fgmres(const spinor& phi, const spinor& /*x0*/, spinor& x, const bool& print_message = false,
                   const bool /*save_res*/ = false) {
            std::vector<c_double> bf = amg_b200::flatten(phi), xf(bf.size());
            int it = 0;
            amg_b200::check(amg_level_gmres(parent->ctx(), parent->level, amg_b200::dptr(bf), amg_b200::dptr(xf), &it),
                            "GMRES_level_l");
            amg_b200::unflatten(xf, x);
            if (print_message) std::cout << "GMRES on level " << parent->level << ": " << it << " iterations" << std::endl;
            return it;
        }

    private:
        Level* parent;
    };

    Level(int level, std::shared_ptr<amg_b200::Context> const* ctx) : level(level), ctx_(ctx), sap_l(this), gmres_l(this) {}

    void D_operator(const spinor& v, spinor& out) { apply(amg_level_apply, v, out, level, "D_operator"); }
    void P_v(const spinor& v, spinor& out) { apply(amg_prolong, v, out, level, "P_v"); }
    void Pt_v(const spinor& v, spinor& out) { apply(amg_restrict, v, out, level, "Pt_v"); }

    const int level;

private:
    std::shared_ptr<amg_b200::Context> const* ctx_;

public:
    SAP_level_l sap_l;
    GMRES_level_l gmres_l;
    amg_ctx ctx() const { return (*ctx_)->get(); }

private:
    template <typename F>
    void apply(F f, const spinor& v, spinor& out, int l, const char* where) {
        std::vector<c_double> in = amg_b200::flatten(v);
        std::vector<c_double> o(out.empty() ? 0 : out.size() * out[0].size());
        amg_b200::check(f(ctx(), l, amg_b200::dptr(in), amg_b200::dptr(o)), where);
        amg_b200::unflatten(o, out);
    }
};

// ---- AlgebraicMG (include/amg.h:8-91) --------------------------------------------------
class AlgebraicMG {
public:
    AlgebraicMG(const GaugeConf& GConf, const double& m0, const int& nu1, const int& nu2)
        : GConf(GConf), m0(m0), nu1(nu1), nu2(nu2) {
        make_context(AMGV::Nit);
        for (int l = 0; l < AMGV::levels; l++) levels.push_back(std::make_unique<Level>(l, &ctx_));
    }
    // the levels refer to this object's context: neither copied nor moved
    AlgebraicMG(const AlgebraicMG&) = delete;
    AlgebraicMG& operator=(const AlgebraicMG&) = delete;
    // AlgebraicMG::setUpPhase (src/amg.cpp:3-88)
    void setUpPhase(const int& Nit) {
        if (ctx_->nit() != Nit) make_context(Nit);
        amg_b200::check(amg_setup(ctx_->get()), "setUpPhase");
        AMGV::SetUpDone = true;
    }
    // psi_l += cycle applied to eta_l (src/amg.cpp:90-178)
    void v_cycle(const int& l, const spinor& eta_l, spinor& psi_l) { cycle(AMG_CYCLE_V, l, eta_l, psi_l); }
    void k_cycle(const int& l, const spinor& eta_l, spinor& psi_l) { cycle(AMG_CYCLE_K, l, eta_l, psi_l); }
    // AlgebraicMG::applyMultilevel (src/amg.cpp:180-231): repeated cycles as a stand-alone solver
    void applyMultilevel(const int& it, const spinor& rhs, spinor& out, const double tol, const bool print_message) {
        const int n0 = LevelV::Nsites[0], d0 = LevelV::DOF[0];
        spinor Dx(n0, c_vector(d0, 0));
        double norm = 0, err = 0;
        for (const auto& r : rhs)
            for (const auto& v : r) norm += std::norm(v);
        norm = std::sqrt(norm);
        const char* name = AMGV::cycle == 0 ? "V-cycle" : "K-cycle";
        for (int i = 0; i < it; i++) {
            if (AMGV::cycle == 0) v_cycle(0, rhs, out); else k_cycle(0, rhs, out);
            levels[0]->D_operator(out, Dx);
            err = 0;
            for (int n = 0; n < n0; n++)
                for (int d = 0; d < d0; d++) err += std::norm(rhs[n][d] - Dx[n][d]);
            err = std::sqrt(err);
            if (err < tol * norm) {
                if (print_message) std::cout << name << " converged in " << i + 1 << " cycles Error " << err << std::endl;
                return;
            }
        }
        if (print_message) std::cout << name << " did not converge in " << it << " cycles Error " << err << std::endl;
    }

    GaugeConf GConf;
    double m0;
    int nu1, nu2;
    std::vector<std::unique_ptr<Level>> levels;
    amg_ctx ctx() const { return ctx_->get(); }

private:
    std::shared_ptr<amg_b200::Context> ctx_;
    void make_context(int nit) {
        const int s1 = AMGV::nu1, s2 = AMGV::nu2;
        AMGV::nu1 = nu1;
        AMGV::nu2 = nu2;
        ctx_ = std::make_shared<amg_b200::Context>(GConf.Conf, m0, nit);
        AMGV::nu1 = s1;
        AMGV::nu2 = s2;
    }
    void cycle(int kind, int l, const spinor& eta, spinor& psi) {
        std::vector<c_double> e = amg_b200::flatten(eta), p = amg_b200::flatten(psi);
        amg_b200::check(amg_set_cycle(ctx_->get(), kind), "cycle");
        amg_b200::check(amg_cycle(ctx_->get(), l, amg_b200::dptr(e), amg_b200::dptr(p)), "cycle");
        amg_b200::unflatten(p, psi);
    }
};

namespace amg_b200 {
// FGMRES::fgmres (include/fgmres.h:36) on a context's solver: x for D x = phi from x0;
// returns the iteration count k*m + j, or restarts*m if the tolerance was not met
inline int fgmres_on(amg_ctx ctx, const spinor& phi, const spinor& x0, spinor& x, bool print_message, int* status) {
    std::vector<c_double> b = flatten(phi), x0f = flatten(x0), xf(b.size());
    bool zero = true;
    for (const auto& v : x0f) zero = zero && v == c_double(0);
    if (!zero) {  // solve for the correction to x0: D e = b - D x0
        std::vector<c_double> dx(b.size());
        check(amg_dirac_apply(ctx, dptr(x0f), dptr(dx), 1, 0), "fgmres");
        for (size_t i = 0; i < b.size(); i++) b[i] -= dx[i];
    }
    amg_solve_info info{};
    const int st = check(amg_solve(ctx, dptr(b), dptr(xf), 1, &info), "fgmres");
    if (!zero)
        for (size_t i = 0; i < xf.size(); i++) xf[i] += x0f[i];
    unflatten(xf, x);
    if (print_message) {
        if (st == AMG_OK)
            std::cout << "FGMRES converged with " << info.iterations << " iterations, relative residual "
                      << info.rel_residual << std::endl;
        else
            std::cout << "FGMRES did not converge, relative residual " << info.rel_residual << std::endl;
    }
    if (status) *status = st;
    return info.iterations;
}
}  // namespace amg_b200

// ---- FGMRES_AMG (include/amg.h:99-145) -------------------------------------------------
// FGMRES(m, restarts, tol) with D_phi and one AMG cycle (AMGV::cycle) as preconditioner;
// the constructor runs the set-up with AMGV::Nit, as the reference's does.
class FGMRES_AMG {
public:
    FGMRES_AMG(const int& dim1, const int& dim2, const int& m, const int& restarts, const double& tol,
               const GaugeConf& GConf, const double& m0, int precision = AMG_PREC_F64)
        : dim1(dim1), dim2(dim2), GConf(GConf), m0(m0) {
        const int sm = FGMRESV::fgmres_restart_length, sr = FGMRESV::fgmres_restarts;
        const double st = FGMRESV::fgmres_tolerance;
        FGMRESV::fgmres_restart_length = m;
        FGMRESV::fgmres_restarts = restarts;
        FGMRESV::fgmres_tolerance = tol;
        ctx_ = std::make_unique<amg_b200::Context>(GConf.Conf, m0, AMGV::Nit, precision);
        FGMRESV::fgmres_restart_length = sm;
        FGMRESV::fgmres_restarts = sr;
        FGMRESV::fgmres_tolerance = st;
        amg_b200::check(amg_setup(ctx_->get()), "setUpPhase");
        double setup_ms = 0, solve_ms = 0;
        amg_last_timings(ctx_->get(), &setup_ms, &solve_ms);
        std::cout << "Elapsed time for Set-up phase = " << setup_ms / 1e3 << " seconds" << std::endl;
    }
    // FGMRES::fgmres (include/fgmres.h:36): returns the iteration count k*m + j, or
    // restarts*m if the tolerance was not met
    int fgmres(const spinor& phi, const spinor& x0, spinor& x, const bool& print_message = false,
               const bool save_res = false) {
        int st = AMG_OK;
        const int it = amg_b200::fgmres_on(ctx_->get(), phi, x0, x, print_message, &st);
        if (save_res && st == AMG_OK) save_residuals();
        return it;
    }
    amg_ctx ctx() const { return ctx_->get(); }

private:
    int dim1, dim2;
    GaugeConf GConf;
    double m0;
    std::unique_ptr<amg_b200::Context> ctx_;

    // the reference's residual file (src/fgmres.cpp:70-79): "index  |g_{j+1}|" per line
    void save_residuals() {
        int n = 0;
        amg_residual_history(ctx_->get(), nullptr, 0, &n);
        std::vector<double> h(n > 0 ? n : 1);
        amg_residual_history(ctx_->get(), h.data(), n, &n);
        std::ostringstream name;
        name << "Residuals_FGMRES_" << LV::Nx << "x" << LV::Nt << "_Levels" << AMGV::levels
             << (AMGV::cycle == 0 ? "_Vcycle" : "_Kcycle") << ".res";
        std::ofstream f(name.str());
        for (int i = 0; i < n; i++) f << i << std::setw(30) << std::setprecision(17) << std::scientific << h[i] << "\n";
    }
};

// ---- FGMRES_SAP (include/sap.h:194-225) -------------------------------------------------
// FGMRES(m, restarts, tol) with D_phi and one fine-level SAP sweep (nu = 1, z zeroed first)
// as the preconditioner, on SAPV::sap_block_x x SAPV::sap_block_t SAP blocks as the
// reference's global fine-level SAP object uses them.  The context still runs its set-up,
// which owns the SAP work buffers.
class FGMRES_SAP {
public:
    FGMRES_SAP(const int& dim1, const int& dim2, const int& m, const int& restarts, const double& tol,
               const c_matrix& U, const double& m0, int precision = AMG_PREC_F64)
        : dim1(dim1), dim2(dim2), m0(m0) {
        const int sm = FGMRESV::fgmres_restart_length, sr = FGMRESV::fgmres_restarts;
        const double st = FGMRESV::fgmres_tolerance;
        const int sbx = LevelV::SAP_Block_x[0], sbt = LevelV::SAP_Block_t[0];
        FGMRESV::fgmres_restart_length = m;
        FGMRESV::fgmres_restarts = restarts;
        FGMRESV::fgmres_tolerance = tol;
        LevelV::SAP_Block_x[0] = SAPV::sap_block_x;
        LevelV::SAP_Block_t[0] = SAPV::sap_block_t;
        ctx_ = std::make_unique<amg_b200::Context>(U, m0, 0, precision);
        FGMRESV::fgmres_restart_length = sm;
        FGMRESV::fgmres_restarts = sr;
        FGMRESV::fgmres_tolerance = st;
        LevelV::SAP_Block_x[0] = sbx;
        LevelV::SAP_Block_t[0] = sbt;
        amg_b200::check(amg_setup(ctx_->get()), "FGMRES_SAP");
        amg_b200::check(amg_set_preconditioner(ctx_->get(), AMG_PRECOND_SAP), "FGMRES_SAP");
    }
    // FGMRES::fgmres (include/fgmres.h:36)
    int fgmres(const spinor& phi, const spinor& x0, spinor& x, const bool& print_message = false,
               const bool save_res = false) {
        (void)save_res;
        return amg_b200::fgmres_on(ctx_->get(), phi, x0, x, print_message, nullptr);
    }
    amg_ctx ctx() const { return ctx_->get(); }

private:
    int dim1, dim2;
    double m0;
    std::unique_ptr<amg_b200::Context> ctx_;
};

// ---- FGMRES_fine_level (include/fgmres.h:126-148): GMRES without preconditioning -------
class FGMRES_fine_level {
public:
    FGMRES_fine_level(const int& dim1, const int& dim2, const int& m, const int& restarts, const double& tol,
                      const c_matrix& U, const double& m0)
        : dim1(dim1), dim2(dim2), m0(m0) {
        const int sm = FGMRESV::fgmres_restart_length, sr = FGMRESV::fgmres_restarts;
        const double st = FGMRESV::fgmres_tolerance;
        FGMRESV::fgmres_restart_length = m;
        FGMRESV::fgmres_restarts = restarts;
        FGMRESV::fgmres_tolerance = tol;
        ctx_ = std::make_unique<amg_b200::Context>(U, m0, 0);
        FGMRESV::fgmres_restart_length = sm;
        FGMRESV::fgmres_restarts = sr;
        FGMRESV::fgmres_tolerance = st;
        amg_b200::check(amg_setup(ctx_->get()), "FGMRES_fine_level");
        amg_b200::check(amg_set_preconditioner(ctx_->get(), AMG_PRECOND_NONE), "FGMRES_fine_level");
    }
    // FGMRES::fgmres (include/fgmres.h:36)
    int fgmres(const spinor& phi, const spinor& x0, spinor& x, const bool& print_message = false,
               const bool save_res = false) {
        (void)save_res;
        return amg_b200::fgmres_on(ctx_->get(), phi, x0, x, print_message, nullptr);
    }

private:
    int dim1, dim2;
    double m0;
    std::unique_ptr<amg_b200::Context> ctx_;
};

// ---- conjugate_gradient (include/conjugate_gradient.h:19): x = (D D^dagger)^{-1} phi ----
// from x = phi with CG::max_iter and CG::tol; returns the iteration count at convergence, or
// CG::max_iter when it did not converge (the reference prints a message then)
inline int conjugate_gradient(const c_matrix& U, const spinor& phi, spinor& x, const double& m0) {
    amg_b200::Context ctx(U, m0, 0);
    std::vector<c_double> b = amg_b200::flatten(phi), xf(b.size());
    int it = 0;
    const int st = amg_b200::check(amg_cg_normal(ctx.get(), amg_b200::dptr(b), amg_b200::dptr(xf), CG::max_iter,
                                                 CG::tol, &it),
                                   "conjugate_gradient");
    amg_b200::unflatten(xf, x);
    if (st != AMG_OK) std::cout << "CG did not converge in " << CG::max_iter << " iterations" << std::endl;
    return it;
}

// ---- bi_cgstab (include/bi_cgstab.h:27-29) with func = D_phi ----------------------------
// returns the solution of D x = phi from x0; other operators than D_phi are not offered
inline spinor bi_cgstab(void (*func)(const c_matrix&, const spinor&, spinor&, const double&), const int& dim1,
                        const int& dim2, const c_matrix& U, const c_matrix& phi, const c_matrix& x0, const double& m0,
                        const int& max_iter, const double& tol, const bool& print_message,
                        const bool& save_residuals) {
    (void)save_residuals;
    if (func != &D_phi) throw amg_b200::Error(AMG_ERR_INVALID, "bi_cgstab: only func = D_phi is offered");
    amg_b200::Context ctx(U, m0, 0);
    std::vector<c_double> b = amg_b200::flatten(phi), x0f = amg_b200::flatten(x0), xf(b.size());
    int it = 0;
    const int st = amg_b200::check(amg_bicgstab(ctx.get(), amg_b200::dptr(b), amg_b200::dptr(x0f),
                                                amg_b200::dptr(xf), max_iter, tol, &it),
                                   "bi_cgstab");
    spinor x(dim1, c_vector(dim2, 0));
    amg_b200::unflatten(xf, x);
    if (print_message) {
        if (st == AMG_OK)
            std::cout << "Bi-CG-stab for D converged in " << it << " iterations" << std::endl;
        else
            std::cout << "Bi-CG-stab did not converge in " << max_iter << " iterations" << std::endl;
    }
    return x;
}

#endif
