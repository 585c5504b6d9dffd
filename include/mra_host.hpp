// nonstationary_mra_b200 -- C++ host side of the MRA hot path, source-
// compatible with the reference's interface for that path:
//
//   class Approximation          include/class_approximation.hpp:7-93
//     Approximation(sill, range, nugget, sill_scale, range_scale, nugget_scale)
//     likelihood(), predict(), dump_prediction_result(), loglikelihood,
//     posteriorPredictionMean / posteriorPredictionVariance (per finest region)
//   class Nonstationary_covariance  include/class_nonstationary_covariance.hpp:8-68
//     get_sigmasq / get_beta / get_tausq
//   evaluate_cross_covariance / evaluate_variance_covariance /
//   evaluate_nonstationary_cross_covariance /
//   evaluate_nonstationary_variance_covariance
//                                include/evaluate_covariance.hpp:25,47,71,88
//   read_user_parameters()       include/read_user_parameters.hpp:3
//   get_optimal_parameters() / get_optimal_nonstationary_parameters()
//                                include/optimization.hpp:1-4
//
// The reference keeps its configuration and data in globals
// (include/constants.hpp:12-205); here they live in one process-wide
// mra_host::Session, filled by read_user_parameters() and load_session()
// (the work of src/main.cpp:93-113: data, fields, partition), which keeps the
// partition resident on the GPU across Approximation objects.  Compute goes
// through the C ABI (mra_b200.h); nothing here runs on the CPU besides file
// IO and the partition builder.  Errors print the reference's style of
// message and exit(EXIT_FAILURE), as the reference does.
#ifndef MRA_HOST_HPP
#define MRA_HOST_HPP

#include <map>
#include <string>
#include <vector>

#include "mra_b200.h"

namespace mra_host {

// KEY=value pairs of user_parameters (and of the optional ext_parameters
// file with the extension keys MRA_EXT_PLANAR, MRA_EXT_NU_X2,
// MRA_EXT_PREFACTOR_EXP, MRA_EXT_BASIS, MRA_EXT_PRECISION).
struct Parameters {
    std::map<std::string, std::string> kv;
    std::string get(const std::string& key, const std::string& def = "") const;
    bool flag(const std::string& key, bool def = false) const;
    double num(const std::string& key, double def) const;
};

// Parses a file in the reference's format (read_user_parameters.cpp:10-50):
// leading spaces/tabs skipped, '#' comment lines, spaces, tabs and quotes
// dropped, everything after the first '=' is the value (further '=' dropped).
Parameters parse_parameter_file(const std::string& path, bool required);

// Flat partition, ready for mra_create.
struct Structure {
    int J = 0, M = 0, r = 0;
    uint64_t n_interior = 0, n_finest = 0;
    std::vector<uint64_t> finest_parent;
    std::vector<double> knots;     // [3][n_interior r]
    std::vector<uint64_t> obs_offset;
    std::vector<double> obs;       // [3][n_obs]
    std::vector<double> obs_value;
    std::vector<uint64_t> obs_index;
    std::vector<uint64_t> pred_offset;
    std::vector<double> pred;      // [3][n_pred]
    std::vector<double> pred_lon, pred_lat;  // prediction locations in dump order
    bool has_pred = false;
    uint64_t n_obs() const { return obs_value.size(); }
};

struct FieldData {
    double intercept = 0;
    std::vector<double> centers;   // [3][nb]
    std::vector<double> weights;
};

struct Session {
    std::string dir = ".";
    Parameters P, X;
    std::string mode;              // CALCULATION_MODE
    Structure st;
    mra_model model{};
    FieldData fields[3];
    int precision = MRA_PRECISION_FP64;
    mra_ctx* ctx = nullptr;
    bool verbose = true;
};

Session& session();

// Loads data, fields and partition for the session's parameters (the work of
// src/main.cpp:93-113) and, unless with_device is false, creates the device
// context.
void load_session(const std::string& dir = ".", bool with_device = true);

// Writes the session's structure in a flat binary form (u64 J, M, r,
// n_interior, n_finest, n_obs, n_pred; then finest_parent, knots [3][.],
// obs_offset, obs [3][.], obs_value, pred_offset, pred [3][.]) for tests.
void dump_structure(const std::string& path);
void close_session();

// Partition built by program (class_partition.cpp:459-654).
Structure build_by_program(const std::vector<double>& lon, const std::vector<double>& lat,
                           const std::vector<double>& val, const std::vector<double>& all_lon,
                           const std::vector<double>& all_lat, int J, int M, int r_requested, double offset,
                           const std::vector<double>* pred_lon, const std::vector<double>* pred_lat, int distance);

// The reference's prediction dump (class_approximation.cpp:493-535).
void write_prediction_dump(const std::string& path, const std::vector<double>& lon, const std::vector<double>& lat,
                           const std::vector<double>& mean, const std::vector<double>& var);

}  // namespace mra_host

// Reads ./user_parameters (and ./ext_parameters when present) into the session.
void read_user_parameters();

class Approximation {
  public:
    Approximation(double sill, double range, double nugget, double sill_scale, double range_scale,
                  double nugget_scale);
    ~Approximation();
    Approximation(const Approximation&) = delete;
    Approximation& operator=(const Approximation&) = delete;

    // Prior + posterior; loglikelihood receives the reference's internal value
    // d (log-determinants plus quadratic forms, without -1/2 and the constant).
    void likelihood();
    // Posterior prediction at the session's prediction locations.
    void predict();
    void dump_prediction_result();

    double loglikelihood = 0.0;
    std::vector<double>* posteriorPredictionMean = nullptr;      // [n_finest]
    std::vector<double>* posteriorPredictionVariance = nullptr;  // [n_finest]

  private:
    mra_theta theta_{};
    void apply_theta();
};

class Nonstationary_covariance {
  public:
    // Fields of the session's model (basis files loaded by load_session).
    double get_sigmasq(double lon, double lat) const;
    double get_beta(double lon, double lat) const;
    double get_tausq(double lon, double lat) const;

  private:
    double field(int f, double lon, double lat) const;
};

// Covariance blocks, out[i1 * n2 + i2] (evaluate_covariance.cpp:56-313).  The
// coordinate arguments are those of the reference; (x, y, z) are used for
// chordal distance, (lon, lat) otherwise.
void evaluate_cross_covariance(double* out, double* lon1, double* lat1, double* x1, double* y1, double* z1,
                               double* lon2, double* lat2, double* x2, double* y2, double* z2,
                               const unsigned long& n1, const unsigned long& n2, const double& sill,
                               const double& range, const double& nugget);
void evaluate_variance_covariance(double* out, double* lon, double* lat, double* x, double* y, double* z,
                                  const unsigned long& n, const double& sill, const double& range,
                                  const double& nugget);
void evaluate_nonstationary_cross_covariance(double* out, double* lon1, double* lat1, double* x1, double* y1,
                                             double* z1, double* lon2, double* lat2, double* x2, double* y2,
                                             double* z2, const unsigned long& n1, const unsigned long& n2,
                                             const double& sill_scale, const double& range_scale,
                                             const double& nugget_scale);
void evaluate_nonstationary_variance_covariance(double* out, double* lon, double* lat, double* x, double* y,
                                                double* z, const unsigned long& n, const double& sill_scale,
                                                const double& range_scale, const double& nugget_scale);

// CALCULATION_MODE=optimization (src/optimization.cpp:66-192): minimises the
// internal loglikelihood over (sill, range, nugget) or over the three scales
// with the library's bound-constrained trust-region optimizer.
void get_optimal_parameters();
void get_optimal_nonstationary_parameters();

#endif  // MRA_HOST_HPP
