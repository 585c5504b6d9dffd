/*
 * CPU-oracle driver for the reference MRA (test infrastructure only).
 *
 * Links against the reference's own, unmodified sources (constants.cpp,
 * read_user_parameters.cpp, class_data.cpp, class_nonstationary_covariance.cpp,
 * class_partition.cpp, evaluate_covariance.cpp, class_approximation*.cpp) and
 * replaces only src/main.cpp, whose flow it follows (src/main.cpp:93-148):
 * read ./user_parameters, load data, load the nonstationary model, build the
 * partition, then run Approximation::likelihood() (and predict() +
 * dump_prediction_result() in prediction mode).  Differences from main.cpp:
 *   - the internal quantity d (Approximation::loglikelihood after
 *     likelihood(), src/class_approximation-posterior-inference.cpp:232-246)
 *     and the final log-likelihood are printed with 17 significant digits;
 *   - `--reps K` evaluates the likelihood K times, each on a fresh
 *     Approximation after resetting the working-region flags exactly as the
 *     reference's optimizer objective does (src/optimization.cpp:121-141),
 *     and prints the wall time of each likelihood() call;
 *   - `--dump-state DIR` (prediction mode) writes the posterior factors per
 *     interior region as raw doubles for kernel-level comparisons.
 * Reference progress prints go to stdout as usual; harness results are
 * printed on lines starting with "ORACLE ".
 */
#include <sys/time.h>
#include <omp.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <armadillo>
#include <mpi.h>

#include "class_data.hpp"
#include "class_nonstationary_covariance.hpp"
#include "class_partition.hpp"
#include "constants.hpp"
#include "read_user_parameters.hpp"
// Opened up only so the harness can read the posterior factors for dumps.
#define private public
#include "class_approximation.hpp"
#undef private

static double now_s() {
    timeval t;
    gettimeofday(&t, nullptr);
    return (double)t.tv_sec + 1e-6 * (double)t.tv_usec;
}

// Mirrors src/optimization.cpp:121-141: restore the working-region state that
// posterior_inference() consumes, so that likelihood() can run again.
static void reset_working_regions() {
    INDICES_REGIONS_AT_CURRENT_LEVEL.clear();
    for (unsigned long iRegion = REGION_START[NUM_LEVELS_M - 1]; iRegion < REGION_END[NUM_LEVELS_M - 1] + 1; iRegion++) {
        unsigned long ancestor = iRegion;
        WORKING_REGION_FLAG[ancestor] = true;
        if (VARIOUS_J_FINEST_LEVEL_FLAG)
            ancestor = partition->parent[iRegion - partition->indexStartFinestLevel];
        else
            ancestor = (iRegion - 1) / NUM_PARTITIONS_J;
        INDICES_REGIONS_AT_CURRENT_LEVEL.insert(ancestor);
        WORKING_REGION_FLAG[ancestor] = true;
        while (ancestor > 0) {
            ancestor = (ancestor - 1) / NUM_PARTITIONS_J;
            WORKING_REGION_FLAG[ancestor] = true;
        }
    }
}

static void write_raw(const std::string& path, const double* p, size_t n) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) {
        std::fprintf(stderr, "cannot write %s\n", path.c_str());
        std::exit(2);
    }
    if (n) std::fwrite(p, sizeof(double), n, f);
    std::fclose(f);
}

int main(int argc, char** argv) {
    int reps = 1;
    std::string dump_dir;
    for (int i = 1; i < argc; ++i) {
        if (!std::strcmp(argv[i], "--reps") && i + 1 < argc) reps = std::atoi(argv[++i]);
        else if (!std::strcmp(argv[i], "--dump-state") && i + 1 < argc) dump_dir = argv[++i];
        else {
            std::fprintf(stderr, "usage: %s [--reps K] [--dump-state DIR]\n", argv[0]);
            return 2;
        }
    }
    gettimeofday(&timeBegin, nullptr);
    int provided = 0;
    MPI_Init_thread(&argc, &argv, MPI_THREAD_MULTIPLE, &provided);
    MPI_Comm_size(MPI_COMM_WORLD, &MPI_SIZE);
    MPI_Comm_rank(MPI_COMM_WORLD, &WORKER);

    read_user_parameters();
    data = new Data;
    data->load_data();
    if (NONSTATIONARY_FLAG) {
        nonstat_cov = new Nonstationary_covariance;
        nonstat_cov->load_data();
    }
    partition = new Partition;
    partition->build_partition();

    std::printf("ORACLE threads=%d n_obs=%lu n_pred=%lu M=%d J=%d r=%d regions=%lu\n", omp_get_max_threads(),
                NUM_OBSERVATIONS, NUM_PREDICTIONS, NUM_LEVELS_M, NUM_PARTITIONS_J, partition->nKnots,
                partition->nRegionsInTotal);

    if (CALCULATION_MODE == "likelihood") {
        for (int rep = 0; rep < reps; ++rep) {
            if (rep > 0) reset_working_regions();
            Approximation approximation(SIGMASQ, BETA, TAUSQ, SIGMASQ_SCALE, BETA_SCALE, TAUSQ_SCALE);
            double t0 = now_s();
            approximation.likelihood();
            double t1 = now_s();
            double d = approximation.loglikelihood;
            double ll = -0.5 * (d + NUM_OBSERVATIONS * std::log(2 * 3.14159265359));
            std::printf("ORACLE rep=%d likelihood_seconds=%.6f d=%.17g loglik=%.17g\n", rep, t1 - t0, d, ll);
        }
    } else if (CALCULATION_MODE == "prediction") {
        Approximation approximation(SIGMASQ, BETA, TAUSQ, SIGMASQ_SCALE, BETA_SCALE, TAUSQ_SCALE);
        double t0 = now_s();
        approximation.likelihood();
        double t1 = now_s();
        approximation.predict();
        double t2 = now_s();
        std::printf("ORACLE likelihood_seconds=%.6f predict_seconds=%.6f\n", t1 - t0, t2 - t1);
        if (DUMP_PREDICTION_RESULTS_FLAG) approximation.dump_prediction_result();
        if (!dump_dir.empty()) {
            const int r = partition->nKnots;
            unsigned long nInterior = partition->nRegionsInTotal - partition->nRegionsAtEachLevel[NUM_LEVELS_M - 1];
            // Posterior Cholesky factors (RChol is overwritten by the posterior pass)
            // and v = L~^{-1} w for every interior region, region-major.
            std::vector<double> L((size_t)nInterior * r * r), v((size_t)nInterior * r);
            for (unsigned long i = 0; i < nInterior; ++i) {
                std::memcpy(&L[(size_t)i * r * r], approximation.RChol[i].memptr(), sizeof(double) * r * r);
                std::memcpy(&v[(size_t)i * r], approximation.KCholTimesCurrentw[i].memptr(), sizeof(double) * r);
            }
            write_raw(dump_dir + "/posterior_L.bin", L.data(), L.size());
            write_raw(dump_dir + "/posterior_v.bin", v.data(), v.size());
        }
    } else {
        std::fprintf(stderr, "oracle harness supports CALCULATION_MODE likelihood or prediction only\n");
        return 2;
    }
    std::fflush(stdout);
    return 0;
}
