// Drop-in executable for the reference's MRA program (src/main.cpp:93-145):
// run in a directory holding user_parameters (and the data files it names),
// it performs CALCULATION_MODE = build_structure_only | likelihood |
// prediction | optimization on one GPU.  An optional argument names the
// directory instead of the current one; `--dump-structure FILE` writes the
// partition (mra_host::dump_structure) and stops before touching the GPU.
#include <cstdio>
#include <iostream>
#include <string>

#include "../../include/mra_host.hpp"

int main(int argc, char** argv) {
    std::string dir = ".", dump;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--dump-structure" && i + 1 < argc) dump = argv[++i];
        else dir = a;
    }
    mra_host::Session& S = mra_host::session();
    S.P = mra_host::parse_parameter_file(dir == "." ? "user_parameters" : dir + "/user_parameters", true);
    S.X = mra_host::parse_parameter_file(dir == "." ? "ext_parameters" : dir + "/ext_parameters", false);
    if (!dump.empty()) {
        mra_host::load_session(dir, false);
        mra_host::dump_structure(dump);
        return 0;
    }
    mra_host::load_session(dir);
    const mra_host::Structure& st = S.st;
    const std::string& mode = S.mode;
    const double sill = S.P.num("SIGMASQ", 1), range = S.P.num("BETA", 1), nugget = S.P.num("TAUSQ", 0);
    const double ss = S.P.num("SIGMASQ_SCALE", 1), rs = S.P.num("BETA_SCALE", 1), ns = S.P.num("TAUSQ_SCALE", 1);
    if (mode == "build_structure_only") {
        std::cout << "Structure: J=" << st.J << " M=" << st.M << " r=" << st.r << " interior regions " << st.n_interior
                  << ", finest regions " << st.n_finest << ", observations " << st.n_obs() << std::endl;
    }
    if (mode == "likelihood") {
        Approximation a(sill, range, nugget, ss, rs, ns);
        a.likelihood();
        std::printf("d=%.17g\n", a.loglikelihood);
    }
    if (mode == "prediction") {
        Approximation a(sill, range, nugget, ss, rs, ns);
        a.likelihood();
        std::printf("d=%.17g\n", a.loglikelihood);
        a.predict();
        if (S.P.flag("DUMP_PREDICTION_RESULTS_FLAG")) a.dump_prediction_result();
    }
    if (mode == "optimization") {
        if (S.P.flag("NONSTATIONARY_FLAG")) get_optimal_nonstationary_parameters();
        else get_optimal_parameters();
    }
    mra_host::close_session();
    return 0;
}
