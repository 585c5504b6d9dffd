// C++ host side of the MRA hot path (include/mra_host.hpp): the reference's
// user_parameters file, its binary data / basis / knots / parent formats, the
// partition, and the Approximation / Nonstationary_covariance /
// evaluate_*covariance interface, over the C ABI of libmra_b200.so.
#include "../../include/mra_host.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <iterator>
#include <unordered_map>

#include "../../include/mra_surrogate.h"

namespace mra_host {

namespace {

Session g_session;

[[noreturn]] void die(const std::string& msg) {
    std::cout << "Program exits with an error: " << msg << std::endl;
    close_session();
    std::exit(EXIT_FAILURE);
}

void check(mra_status s, const char* where) {
    if (s != MRA_OK) die(std::string(where) + " failed: " + mra_last_error());
}

std::vector<char> read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) die("fail to open the data file " + path);
    return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

// Sequential reader of the reference's binary files (u64 counts, f64 values).
struct Reader {
    std::vector<char> raw;
    size_t off = 0;
    std::string path;
    explicit Reader(const std::string& p) : raw(read_file(p)), path(p) {}
    void need(size_t bytes, const char* what) const {
        if (off + bytes > raw.size())
            die(std::string("fail reading data file ") + path + " for " + what +
                ". Double check the data file format.");
    }
    uint64_t u64(const char* what) {
        need(8, what);
        uint64_t v;
        std::memcpy(&v, raw.data() + off, 8);
        off += 8;
        return v;
    }
    std::vector<double> f64s(size_t n, const char* what) {
        need(8 * n, what);
        std::vector<double> v(n);
        std::memcpy(v.data(), raw.data() + off, 8 * n);
        off += 8 * n;
        return v;
    }
    std::vector<uint64_t> u64s(size_t n, const char* what) {
        need(8 * n, what);
        std::vector<uint64_t> v(n);
        std::memcpy(v.data(), raw.data() + off, 8 * n);
        off += 8 * n;
        return v;
    }
};

uint64_t n_interior_of(int J, int M) {
    uint64_t s = 0, p = 1;
    for (int m = 0; m < M - 1; ++m) s += p, p *= (uint64_t)J;
    return s;
}

// lon/lat -> the coordinates the device uses for the distance kind
void coords_of(const std::vector<double>& lon, const std::vector<double>& lat, int distance,
               std::vector<double>& out) {
    const size_t n = lon.size();
    out.assign(3 * n, 0.0);
    for (size_t i = 0; i < n; ++i) {
        if (distance == MRA_DIST_CHORDAL) {
            // class_partition.cpp:262-270, degrees as (deg * pi) / 180
            double la = lat[i] * M_PI / 180, lo = lon[i] * M_PI / 180;
            out[i] = std::cos(la) * std::cos(lo);
            out[n + i] = std::cos(la) * std::sin(lo);
            out[2 * n + i] = std::sin(la);
        } else {
            out[i] = lon[i];
            out[n + i] = lat[i];
        }
    }
}

struct Boxes {
    std::vector<double> lo0, hi0, lo1, hi1;
};

// region boxes in heap order: class_partition.cpp:49-88,476-490, domain from
// class_data.cpp:150-165
Boxes make_boxes(int J, int M, const std::vector<double>& all_lon, const std::vector<double>& all_lat) {
    const uint64_t n_int = n_interior_of(J, M);
    uint64_t n_fin = 1;
    for (int m = 0; m < M - 1; ++m) n_fin *= (uint64_t)J;
    const uint64_t n_tot = n_int + n_fin;
    Boxes b;
    b.lo0.resize(n_tot);
    b.hi0.resize(n_tot);
    b.lo1.resize(n_tot);
    b.hi1.resize(n_tot);
    const double mnx = *std::min_element(all_lon.begin(), all_lon.end());
    const double mxx = *std::max_element(all_lon.begin(), all_lon.end());
    const double mny = *std::min_element(all_lat.begin(), all_lat.end());
    const double mxy = *std::max_element(all_lat.begin(), all_lat.end());
    b.lo0[0] = mnx;
    b.hi0[0] = mxx + 1e-6 * (mxx - mnx);
    b.lo1[0] = mny;
    b.hi1[0] = mxy + 1e-6 * (mxy - mny);
    uint64_t s = 0, cnt = 1;
    for (int m = 0; m < M - 1; ++m) {
        for (uint64_t reg = s; reg < s + cnt; ++reg) {
            const double a = b.lo0[reg], bb = b.hi0[reg], c = b.lo1[reg], d = b.hi1[reg];
            if (J == 2) {
                const bool split_lon = (bb - a) >= (d - c);
                const double mid_lon = (bb + a) / 2, mid_lat = (d + c) / 2;
                const uint64_t c1 = 2 * reg + 1, c2 = 2 * reg + 2;
                b.lo0[c1] = a;
                b.hi0[c1] = split_lon ? mid_lon : bb;
                b.lo0[c2] = split_lon ? mid_lon : a;
                b.hi0[c2] = bb;
                b.lo1[c1] = c;
                b.hi1[c1] = split_lon ? d : mid_lat;
                b.lo1[c2] = split_lon ? c : mid_lat;
                b.hi1[c2] = d;
            } else {
                const double lm = (bb + a) / 2, tm = (d + c) / 2;
                const uint64_t ch = 4 * reg;
                const double l0[4] = {a, lm, a, lm}, h0[4] = {lm, bb, lm, bb};
                const double l1[4] = {c, c, tm, tm}, h1[4] = {tm, tm, d, d};
                for (int k = 0; k < 4; ++k) {
                    b.lo0[ch + 1 + k] = l0[k];
                    b.hi0[ch + 1 + k] = h0[k];
                    b.lo1[ch + 1 + k] = l1[k];
                    b.hi1[ch + 1 + k] = h1[k];
                }
            }
        }
        s += cnt;
        cnt *= (uint64_t)J;
    }
    return b;
}

// finest index of a point (-1: outside every box), descending the tree with the
// reference's containment test lo <= p < hi
int64_t finest_of(int J, int M, const Boxes& b, double lon, double lat) {
    uint64_t idx = 0;
    for (int m = 0; m < M - 1; ++m) {
        int64_t nxt = -1;
        for (int c = 1; c <= J; ++c) {
            const uint64_t ch = idx * J + c;
            if (lon >= b.lo0[ch] && lon < b.hi0[ch] && lat >= b.lo1[ch] && lat < b.hi1[ch]) {
                nxt = (int64_t)ch;
                break;
            }
        }
        if (nxt < 0) return -1;
        idx = (uint64_t)nxt;
    }
    return (int64_t)(idx - n_interior_of(J, M));
}

// stable counting sort of rows by finest index: (order, CSR offsets)
void csr(const std::vector<int64_t>& fidx, const std::vector<uint64_t>& rows, uint64_t n_fin,
         std::vector<uint64_t>& order, std::vector<uint64_t>& off) {
    off.assign(n_fin + 1, 0);
    for (uint64_t r : rows) off[fidx[r] + 1]++;
    for (uint64_t k = 0; k < n_fin; ++k) off[k + 1] += off[k];
    std::vector<uint64_t> pos(off.begin(), off.end() - 1);
    order.assign(rows.size(), 0);
    for (uint64_t r : rows) order[pos[fidx[r]]++] = r;
}

struct PairHash {
    size_t operator()(const std::pair<uint64_t, uint64_t>& p) const {
        return (size_t)(p.first * 0x9E3779B97F4A7C15ull ^ p.second);
    }
};

std::pair<uint64_t, uint64_t> key_of(double lon, double lat) {
    uint64_t a, b;
    std::memcpy(&a, &lon, 8);
    std::memcpy(&b, &lat, 8);
    return {a, b};
}

FieldData load_basis(const std::string& path, int distance) {
    Reader rd(path);
    const uint64_t m = rd.u64("the number of basis functions");
    FieldData f;
    f.intercept = rd.f64s(1, "the intercept")[0];
    std::vector<double> lon = rd.f64s(m, "basis longitudes"), lat = rd.f64s(m, "basis latitudes");
    f.weights = rd.f64s(m, "basis weights");
    coords_of(lon, lat, distance, f.centers);
    return f;
}

std::string path_in(const std::string& dir, const std::string& name) {
    if (name.empty() || name[0] == '/' || dir.empty() || dir == ".") return name;
    return dir + "/" + name;
}

// rows (in the given order) -> the structure's sorted observation or
// prediction arrays
void take_rows(const std::vector<uint64_t>& order, const std::vector<double>& lon, const std::vector<double>& lat,
               std::vector<double>& olon, std::vector<double>& olat) {
    olon.resize(order.size());
    olat.resize(order.size());
    for (size_t k = 0; k < order.size(); ++k) {
        olon[k] = lon[order[k]];
        olat[k] = lat[order[k]];
    }
}

// PROVIDED_KNOTS_FLAG with the finest parents from a file:
// class_partition.cpp:93-454, 659-770
Structure build_by_user_files(const std::vector<double>& lon, const std::vector<double>& lat,
                              const std::vector<double>& val, const std::vector<uint64_t>& obs_region, int J, int M,
                              int r, const std::string& knots_path, const std::string& parent_path,
                              const std::vector<double>* pred_lon, const std::vector<double>* pred_lat,
                              const std::vector<uint64_t>* pred_region, int distance) {
    Structure st;
    st.J = J;
    st.M = M;
    st.r = r;
    st.n_interior = n_interior_of(J, M);
    const uint64_t n_int = st.n_interior;
    Reader kr(knots_path);
    const uint64_t k = kr.u64("the number of knots");
    std::vector<double> kl = kr.f64s(k, "knot longitudes"), kt = kr.f64s(k, "knot latitudes");
    std::vector<uint64_t> kreg = kr.u64s(k, "knot regions");
    Reader pr(parent_path);
    const uint64_t start = pr.u64("the first finest region"), end = pr.u64("the last finest region");
    if (start != n_int) die("the first finest region of the parent file must follow the interior regions");
    st.finest_parent = pr.u64s(end - start + 1, "parent region indices");
    st.n_finest = st.finest_parent.size();
    std::vector<double> klon(n_int * r, 0.0), klat(n_int * r, 0.0);
    for (uint64_t i = 0; i < k && kreg[i] < n_int;) {  // class_partition.cpp:247-276
        const uint64_t reg = kreg[i];
        for (int q = 0; q < r && i + q < k; ++q) {
            klon[reg * r + q] = kl[i + q];
            klat[reg * r + q] = kt[i + q];
        }
        i += r;
    }
    coords_of(klon, klat, distance, st.knots);
    std::vector<int64_t> fidx(obs_region.size());
    std::vector<uint64_t> rows(obs_region.size());
    for (size_t t = 0; t < obs_region.size(); ++t) {
        if (obs_region[t] < n_int || obs_region[t] >= n_int + st.n_finest)
            die("observation region index outside the finest level");
        fidx[t] = (int64_t)(obs_region[t] - n_int);
        rows[t] = t;
    }
    csr(fidx, rows, st.n_finest, st.obs_index, st.obs_offset);
    std::vector<double> olon, olat;
    take_rows(st.obs_index, lon, lat, olon, olat);
    st.obs_value.resize(st.obs_index.size());
    for (size_t q = 0; q < st.obs_index.size(); ++q) st.obs_value[q] = val[st.obs_index[q]];
    coords_of(olon, olat, distance, st.obs);
    if (pred_lon) {
        std::vector<int64_t> pidx(pred_lon->size());
        std::vector<uint64_t> prow(pred_lon->size()), porder;
        for (size_t t = 0; t < pred_lon->size(); ++t) {
            if ((*pred_region)[t] < n_int || (*pred_region)[t] >= n_int + st.n_finest)
                die("prediction region index outside the finest level");
            pidx[t] = (int64_t)((*pred_region)[t] - n_int);
            prow[t] = t;
        }
        csr(pidx, prow, st.n_finest, porder, st.pred_offset);
        take_rows(porder, *pred_lon, *pred_lat, st.pred_lon, st.pred_lat);
        coords_of(st.pred_lon, st.pred_lat, distance, st.pred);
        st.has_pred = true;
    }
    return st;
}

}  // namespace

// ---------------------------------------------------------------------------
// parameters
// ---------------------------------------------------------------------------
std::string Parameters::get(const std::string& key, const std::string& def) const {
    auto it = kv.find(key);
    return it == kv.end() ? def : it->second;
}
bool Parameters::flag(const std::string& key, bool def) const {
    auto it = kv.find(key);
    if (it == kv.end()) return def;
    return it->second == "true" || it->second == "TRUE" || it->second == "True";
}
double Parameters::num(const std::string& key, double def) const {
    auto it = kv.find(key);
    return it == kv.end() ? def : std::atof(it->second.c_str());
}

Parameters parse_parameter_file(const std::string& path, bool required) {
    Parameters P;
    std::ifstream file(path);
    if (!file) {
        if (required) die("fail to open the parameter file " + path);
        return P;
    }
    std::string line;
    while (std::getline(file, line)) {
        size_t i = 0;
        while (i < line.size() && (line[i] == ' ' || line[i] == '\t')) ++i;
        if (i >= line.size() || line[i] == '#' || line[i] == '\r') continue;
        std::string name, value;
        bool in_name = true;
        for (size_t k = i; k < line.size(); ++k) {
            const char ch = line[k];
            if (ch == ' ' || ch == '\t' || ch == '\'' || ch == '"' || ch == '\r') continue;
            if (ch == '=') {
                in_name = false;
                continue;
            }
            (in_name ? name : value) += ch;
        }
        if (!name.empty()) P.kv[name] = value;
    }
    return P;
}

Session& session() { return g_session; }

// ---------------------------------------------------------------------------
// partition by program
// ---------------------------------------------------------------------------
Structure build_by_program(const std::vector<double>& lon, const std::vector<double>& lat,
                           const std::vector<double>& val, const std::vector<double>& all_lon,
                           const std::vector<double>& all_lat, int J, int M, int r_requested, double offset,
                           const std::vector<double>* pred_lon, const std::vector<double>* pred_lat, int distance) {
    if (J != 2 && J != 4) die("NUM_PARTITIONS_J must be 2 or 4");
    if (M < 2) die("NUM_LEVELS_M must be at least 2");
    if (all_lon.empty()) die("no locations in the data file");
    Structure st;
    st.J = J;
    st.M = M;
    st.n_interior = n_interior_of(J, M);
    st.n_finest = 1;
    for (int m = 0; m < M - 1; ++m) st.n_finest *= (uint64_t)J;
    const uint64_t n_int = st.n_interior, n_fin = st.n_finest;
    const Boxes b = make_boxes(J, M, all_lon, all_lat);
    // knots: create_knots, class_partition.cpp:24-44
    const int nlon = (int)std::ceil(std::sqrt((double)r_requested));
    const int nlat = r_requested / nlon;
    const int r = nlon * nlat;
    st.r = r;
    std::vector<double> klon(n_int * r), klat(n_int * r);
    for (uint64_t reg = 0; reg < n_int; ++reg) {
        const double a = b.lo0[reg], bb = b.hi0[reg], c = b.lo1[reg], d = b.hi1[reg];
        const double off_lon = (bb - a) * offset, off_lat = (d - c) * offset;
        const double lon_start = a + off_lon, lon_end = bb - off_lon;
        const double lat_start = c + off_lat, lat_end = d - off_lat;
        const double lon_inc = nlon == 1 ? 0.0 : (lon_end - lon_start) / (nlon - 1);
        const double lat_inc = nlat == 1 ? 0.0 : (lat_end - lat_start) / (nlat - 1);
        for (int i = 0; i < nlon; ++i)
            for (int j = 0; j < nlat; ++j) {
                klon[reg * r + i * nlat + j] = lon_end - (double)(nlon - i - 1) * lon_inc;
                klat[reg * r + i * nlat + j] = lat_end - (double)(nlat - j - 1) * lat_inc;
            }
    }
    // observations: finest box, minus those that coincide with a knot of an
    // ancestor (class_partition.cpp:533-551)
    const size_t n = lon.size();
    std::vector<int64_t> fidx(n);
    std::unordered_map<std::pair<uint64_t, uint64_t>, std::vector<uint64_t>, PairHash> knot_regions;
    for (uint64_t q = 0; q < n_int * (uint64_t)r; ++q) knot_regions[key_of(klon[q], klat[q])].push_back(q / r);
    std::vector<uint64_t> rows;
    rows.reserve(n);
    for (size_t t = 0; t < n; ++t) {
        fidx[t] = finest_of(J, M, b, lon[t], lat[t]);
        if (fidx[t] < 0) continue;
        bool keep = true;
        auto it = knot_regions.find(key_of(lon[t], lat[t]));
        if (it != knot_regions.end()) {
            uint64_t anc = n_int + (uint64_t)fidx[t];
            for (int m = 0; m < M - 1 && keep; ++m) {
                anc = (anc - 1) / J;
                for (uint64_t reg : it->second)
                    if (reg == anc) keep = false;
            }
        }
        if (keep) rows.push_back(t);
    }
    csr(fidx, rows, n_fin, st.obs_index, st.obs_offset);
    std::vector<double> olon, olat;
    take_rows(st.obs_index, lon, lat, olon, olat);
    st.obs_value.resize(st.obs_index.size());
    for (size_t k = 0; k < st.obs_index.size(); ++k) st.obs_value[k] = val[st.obs_index[k]];
    coords_of(olon, olat, distance, st.obs);
    coords_of(klon, klat, distance, st.knots);
    st.finest_parent.resize(n_fin);
    for (uint64_t k = 0; k < n_fin; ++k) st.finest_parent[k] = (n_int + k - 1) / J;
    if (pred_lon) {
        std::vector<int64_t> pidx(pred_lon->size());
        std::vector<uint64_t> prow, porder;
        for (size_t t = 0; t < pred_lon->size(); ++t) {
            pidx[t] = finest_of(J, M, b, (*pred_lon)[t], (*pred_lat)[t]);
            if (pidx[t] >= 0) prow.push_back(t);
        }
        csr(pidx, prow, n_fin, porder, st.pred_offset);
        take_rows(porder, *pred_lon, *pred_lat, st.pred_lon, st.pred_lat);
        coords_of(st.pred_lon, st.pred_lat, distance, st.pred);
        st.has_pred = true;
    }
    return st;
}

// ---------------------------------------------------------------------------
// session: data, fields, partition, device context
// ---------------------------------------------------------------------------
void load_session(const std::string& dir, bool with_device) {
    Session& S = g_session;
    S.dir = dir;
    if (S.P.kv.empty()) {
        S.P = parse_parameter_file(path_in(dir, "user_parameters"), true);
        S.X = parse_parameter_file(path_in(dir, "ext_parameters"), false);
    }
    const Parameters& P = S.P;
    const Parameters& X = S.X;
    S.mode = P.get("CALCULATION_MODE", "likelihood");
    const bool provided = P.flag("PROVIDED_KNOTS_FLAG");
    const bool chordal = P.flag("CHORDAL_DISTANCE_FLAG", true);
    const int distance = chordal ? MRA_DIST_CHORDAL
                                 : (X.flag("MRA_EXT_PLANAR") ? MRA_DIST_EUCLID2D : MRA_DIST_GREAT_CIRCLE);
    // data: class_data.cpp:47-143 (rows with NaN values are prediction candidates)
    Reader rd(path_in(dir, P.get("DATA_FILE_NAME")));
    const uint64_t n = rd.u64("the number of locations");
    std::vector<double> lon = rd.f64s(n, "longitudes"), lat = rd.f64s(n, "latitudes"), val = rd.f64s(n, "values");
    std::vector<uint64_t> reg;
    if (provided) reg = rd.u64s(n, "region indices");
    std::vector<double> olon, olat, oval, plon, plat;
    std::vector<uint64_t> oreg, preg;
    for (uint64_t i = 0; i < n; ++i) {
        if (std::isnan(val[i])) continue;
        olon.push_back(lon[i]);
        olat.push_back(lat[i]);
        oval.push_back(val[i]);
        if (provided) oreg.push_back(reg[i]);
    }
    const bool want_pred = S.mode == "prediction";
    if (want_pred) {
        const std::string pm = P.get("PREDICTION_LOCATION_MODE", "A");
        if (pm == "A") {
            Reader pr(path_in(dir, P.get("PREDICTION_LOCATION_FILE")));
            const uint64_t np = pr.u64("the number of prediction locations");
            plon = pr.f64s(np, "prediction longitudes");
            plat = pr.f64s(np, "prediction latitudes");
            if (provided) preg = pr.u64s(np, "prediction regions");
        } else {
            for (uint64_t i = 0; i < n; ++i) {
                if (pm == "N" && !std::isnan(val[i])) continue;
                plon.push_back(lon[i]);
                plat.push_back(lat[i]);
                if (provided) preg.push_back(reg[i]);
            }
        }
    }
    const int J = (int)P.num("NUM_PARTITIONS_J", 2), M = (int)P.num("NUM_LEVELS_M", 2);
    const int r = (int)P.num("NUM_KNOTS_r", 1);
    if (provided) {
        S.st = build_by_user_files(olon, olat, oval, oreg, J, M, r, path_in(dir, P.get("KNOTS_FILE_NAME")),
                                   path_in(dir, P.get("PARENT_REGION_FILE_NAME")), want_pred ? &plon : nullptr,
                                   want_pred ? &plat : nullptr, want_pred ? &preg : nullptr, distance);
    } else {
        const std::string off = P.get("OFFSET", "default");
        const double offset = off == "default" ? std::exp(1.0) / 100 : std::atof(off.c_str());
        S.st = build_by_program(olon, olat, oval, lon, lat, J, M, r, offset, want_pred ? &plon : nullptr,
                                want_pred ? &plat : nullptr, distance);
    }
    // covariance model
    mra_model& md = S.model;
    md = mra_model{};
    md.nonstationary = P.flag("NONSTATIONARY_FLAG") ? 1 : 0;
    md.distance = distance;
    md.nu_x2 = (int)X.num("MRA_EXT_NU_X2", 1);
    md.prefactor_exp = X.num("MRA_EXT_PREFACTOR_EXP", 1.5);
    md.dist_scale = distance == MRA_DIST_EUCLID2D ? 1.0 : 6371.0;
    md.basis = X.get("MRA_EXT_BASIS", "wendland") == "gaussian" ? MRA_BASIS_GAUSSIAN : MRA_BASIS_WENDLAND;
    md.basis_len = P.num("WENDLAND_LEN", 0.22);
    if (md.nonstationary) {
        const char* keys[3] = {"SIGMASQ_FILE_NAME", "BETA_FILE_NAME", "TAUSQ_FILE_NAME"};
        for (int f = 0; f < 3; ++f) {
            S.fields[f] = load_basis(path_in(dir, P.get(keys[f])), distance);
            md.field[f].n_basis = S.fields[f].weights.size();
            md.field[f].centers = S.fields[f].centers.data();
            md.field[f].weights = S.fields[f].weights.data();
            md.field[f].intercept = S.fields[f].intercept;
        }
    }
    S.precision = X.get("MRA_EXT_PRECISION", "fp64") == "mixed" ? MRA_PRECISION_MIXED : MRA_PRECISION_FP64;
    if (!with_device) return;
    // device context
    mra_structure s{};
    const Structure& st = S.st;
    s.J = st.J;
    s.M = st.M;
    s.r = st.r;
    s.n_interior = st.n_interior;
    s.n_finest = st.n_finest;
    s.finest_parent = st.finest_parent.data();
    s.knots = st.knots.data();
    s.obs_offset = st.obs_offset.data();
    s.obs = st.obs.data();
    s.obs_value = st.obs_value.data();
    if (st.has_pred) {
        s.pred_offset = st.pred_offset.data();
        s.pred = st.pred.data();
    }
    if (S.ctx) mra_destroy(S.ctx);
    S.ctx = nullptr;
    check(mra_create(&s, &md, S.precision, &S.ctx), "mra_create");
}

void dump_structure(const std::string& path) {
    const Structure& st = g_session.st;
    std::ofstream f(path, std::ios::binary);
    if (!f) die("fail to open the output file " + path);
    auto u = [&](uint64_t v) { f.write(reinterpret_cast<const char*>(&v), 8); };
    auto vu = [&](const std::vector<uint64_t>& v) { f.write(reinterpret_cast<const char*>(v.data()), 8 * v.size()); };
    auto vd = [&](const std::vector<double>& v) { f.write(reinterpret_cast<const char*>(v.data()), 8 * v.size()); };
    const uint64_t np = st.has_pred ? st.pred_offset.back() : 0;
    u(st.J), u(st.M), u(st.r), u(st.n_interior), u(st.n_finest), u(st.n_obs()), u(np);
    vu(st.finest_parent), vd(st.knots), vu(st.obs_offset), vd(st.obs), vd(st.obs_value);
    if (st.has_pred) vu(st.pred_offset), vd(st.pred);
}

void close_session() {
    if (g_session.ctx) mra_destroy(g_session.ctx);
    g_session.ctx = nullptr;
}

void write_prediction_dump(const std::string& path, const std::vector<double>& lon, const std::vector<double>& lat,
                           const std::vector<double>& mean, const std::vector<double>& var) {
    std::ofstream f(path, std::ios::binary);
    if (!f) die("fail to open the output file " + path);
    const uint64_t n = mean.size();
    f.write(reinterpret_cast<const char*>(&n), 8);
    f.write(reinterpret_cast<const char*>(lon.data()), 8 * n);
    f.write(reinterpret_cast<const char*>(lat.data()), 8 * n);
    f.write(reinterpret_cast<const char*>(mean.data()), 8 * n);
    f.write(reinterpret_cast<const char*>(var.data()), 8 * n);
}

}  // namespace mra_host

using namespace mra_host;

void read_user_parameters() {
    Session& S = session();
    S.P = parse_parameter_file("user_parameters", true);
    S.X = parse_parameter_file("ext_parameters", false);
}

// ---------------------------------------------------------------------------
// Approximation
// ---------------------------------------------------------------------------
Approximation::Approximation(double sill, double range, double nugget, double sill_scale, double range_scale,
                             double nugget_scale) {
    theta_.sill = sill;
    theta_.range = range;
    theta_.nugget = nugget;
    theta_.sill_scale = sill_scale;
    theta_.range_scale = range_scale;
    theta_.nugget_scale = nugget_scale;
}

Approximation::~Approximation() {
    delete[] posteriorPredictionMean;
    delete[] posteriorPredictionVariance;
}

void Approximation::apply_theta() {
    Session& S = session();
    if (!S.ctx) load_session(S.dir);
    check(mra_set_theta(S.ctx, &theta_), "mra_set_theta");
}

void Approximation::likelihood() {
    Session& S = session();
    apply_theta();
    double d = 0, ll = 0;
    check(mra_loglik(S.ctx, &d, &ll), "mra_loglik");
    loglikelihood = d;
    if (S.verbose) std::cout << "The obtained loglikelihood is: " << ll << std::endl;
}

void Approximation::predict() {
    Session& S = session();
    apply_theta();
    const Structure& st = S.st;
    if (!st.has_pred) die("no prediction locations (CALCULATION_MODE=prediction loads them)");
    const uint64_t np = st.pred_offset.back();
    std::vector<double> mean(np), var(np);
    check(mra_predict(S.ctx, mean.data(), var.data()), "mra_predict");
    delete[] posteriorPredictionMean;
    delete[] posteriorPredictionVariance;
    posteriorPredictionMean = new std::vector<double>[st.n_finest];
    posteriorPredictionVariance = new std::vector<double>[st.n_finest];
    for (uint64_t k = 0; k < st.n_finest; ++k) {
        posteriorPredictionMean[k].assign(mean.begin() + st.pred_offset[k], mean.begin() + st.pred_offset[k + 1]);
        posteriorPredictionVariance[k].assign(var.begin() + st.pred_offset[k], var.begin() + st.pred_offset[k + 1]);
    }
}

void Approximation::dump_prediction_result() {
    Session& S = session();
    const Structure& st = S.st;
    if (!posteriorPredictionMean) die("dump_prediction_result before predict");
    std::vector<double> mean, var;
    for (uint64_t k = 0; k < st.n_finest; ++k) {
        mean.insert(mean.end(), posteriorPredictionMean[k].begin(), posteriorPredictionMean[k].end());
        var.insert(var.end(), posteriorPredictionVariance[k].begin(), posteriorPredictionVariance[k].end());
    }
    const std::string name = S.P.get("PREDICTION_RESULTS_FILE_NAME", "prediction_results.bin");
    write_prediction_dump(name[0] == '/' || S.dir == "." ? name : S.dir + "/" + name, st.pred_lon, st.pred_lat, mean,
                          var);
}

// ---------------------------------------------------------------------------
// fields and covariance blocks
// ---------------------------------------------------------------------------
double Nonstationary_covariance::field(int f, double lon, double lat) const {
    Session& S = session();
    std::vector<double> p;
    coords_of({lon}, {lat}, S.model.distance, p);
    mra_theta th{};
    th.sill_scale = th.range_scale = th.nugget_scale = 1.0;
    double out[3];
    check(mra_eval_fields(&S.model, &th, p.data(), 1, out), "mra_eval_fields");
    return out[f];
}
double Nonstationary_covariance::get_sigmasq(double lon, double lat) const { return field(0, lon, lat); }
double Nonstationary_covariance::get_beta(double lon, double lat) const { return field(1, lon, lat); }
double Nonstationary_covariance::get_tausq(double lon, double lat) const { return field(2, lon, lat); }

namespace {

std::vector<double> pack_points(const double* lon, const double* lat, const double* x, const double* y,
                                const double* z, unsigned long n, int distance) {
    std::vector<double> p(3 * n, 0.0);
    for (unsigned long i = 0; i < n; ++i) {
        if (distance == MRA_DIST_CHORDAL) {
            p[i] = x[i];
            p[n + i] = y[i];
            p[2 * n + i] = z[i];
        } else {
            p[i] = lon[i];
            p[n + i] = lat[i];
        }
    }
    return p;
}

void cov_call(bool nonstat, double* out, const std::vector<double>& p1, unsigned long n1,
              const std::vector<double>* p2, unsigned long n2, double a, double b, double c) {
    Session& S = session();
    mra_model md = S.model;
    md.nonstationary = nonstat ? 1 : 0;
    mra_theta th{};
    if (nonstat) {
        th.sill_scale = a;
        th.range_scale = b;
        th.nugget_scale = c;
    } else {
        th.sill = a;
        th.range = b;
        th.nugget = c;
        th.sill_scale = th.range_scale = th.nugget_scale = 1.0;
    }
    check(mra_eval_covariance(&md, &th, p1.data(), n1, p2 ? p2->data() : nullptr, p2 ? n2 : 0, p2 ? 0 : 1, out),
          "mra_eval_covariance");
}

}  // namespace

void evaluate_cross_covariance(double* out, double* lon1, double* lat1, double* x1, double* y1, double* z1,
                               double* lon2, double* lat2, double* x2, double* y2, double* z2,
                               const unsigned long& n1, const unsigned long& n2, const double& sill,
                               const double& range, const double& nugget) {
    const int dist = session().model.distance;
    std::vector<double> p1 = pack_points(lon1, lat1, x1, y1, z1, n1, dist);
    std::vector<double> p2 = pack_points(lon2, lat2, x2, y2, z2, n2, dist);
    cov_call(false, out, p1, n1, &p2, n2, sill, range, nugget);
}

void evaluate_variance_covariance(double* out, double* lon, double* lat, double* x, double* y, double* z,
                                  const unsigned long& n, const double& sill, const double& range,
                                  const double& nugget) {
    std::vector<double> p = pack_points(lon, lat, x, y, z, n, session().model.distance);
    cov_call(false, out, p, n, nullptr, 0, sill, range, nugget);
}

void evaluate_nonstationary_cross_covariance(double* out, double* lon1, double* lat1, double* x1, double* y1,
                                             double* z1, double* lon2, double* lat2, double* x2, double* y2,
                                             double* z2, const unsigned long& n1, const unsigned long& n2,
                                             const double& sill_scale, const double& range_scale,
                                             const double& nugget_scale) {
    const int dist = session().model.distance;
    std::vector<double> p1 = pack_points(lon1, lat1, x1, y1, z1, n1, dist);
    std::vector<double> p2 = pack_points(lon2, lat2, x2, y2, z2, n2, dist);
    cov_call(true, out, p1, n1, &p2, n2, sill_scale, range_scale, nugget_scale);
}

void evaluate_nonstationary_variance_covariance(double* out, double* lon, double* lat, double* x, double* y,
                                                double* z, const unsigned long& n, const double& sill_scale,
                                                const double& range_scale, const double& nugget_scale) {
    std::vector<double> p = pack_points(lon, lat, x, y, z, n, session().model.distance);
    cov_call(true, out, p, n, nullptr, 0, sill_scale, range_scale, nugget_scale);
}

// ---------------------------------------------------------------------------
// optimization mode (src/optimization.cpp:66-192)
// ---------------------------------------------------------------------------
namespace {

struct OptState {
    bool nonstat;
    int iteration = 0;
};

double objective(const double* x, void* user, int32_t* /*stop*/) {
    OptState& o = *static_cast<OptState*>(user);
    ++o.iteration;
    Session& S = session();
    if (S.verbose)
        std::cout << "############## Iteration " << o.iteration
                  << (o.nonstat ? ". sigmasq multiplication: " : ". sigmasq: ") << x[0]
                  << (o.nonstat ? ", beta multiplication: " : ", beta: ") << x[1]
                  << (o.nonstat ? ", tausq multiplication: " : ", tausq: ") << x[2] << std::endl;
    double d;
    if (o.nonstat) {
        Approximation a(0.0, 0.0, 0.0, x[0], x[1], x[2]);
        a.likelihood();
        d = a.loglikelihood;
    } else {
        Approximation a(x[0], x[1], x[2], 0.0, 0.0, 0.0);
        a.likelihood();
        d = a.loglikelihood;
    }
    return d;
}

void run_optimization(bool nonstat) {
    Session& S = session();
    const Parameters& P = S.P;
    double x[3], lo[3], hi[3];
    mra_opt_config cfg{};
    cfg.npt = 7;
    cfg.max_evals = (int)P.num("MAX_ITERATIONS", 1000);
    if (nonstat) {
        for (int i = 0; i < 3; ++i) x[i] = 1.0, lo[i] = 1e-2, hi[i] = 1e2;
        cfg.rho_begin = 0.1;
        cfg.rho_end = 1e-6;
    } else {
        const char* g[3] = {"SIGMASQ_INITIAL_GUESS", "BETA_INITIAL_GUESS", "TAUSQ_INITIAL_GUESS"};
        const char* l[3] = {"SIGMASQ_LOWER_BOUND", "BETA_LOWER_BOUND", "TAUSQ_LOWER_BOUND"};
        const char* u[3] = {"SIGMASQ_UPPER_BOUND", "BETA_UPPER_BOUND", "TAUSQ_UPPER_BOUND"};
        for (int i = 0; i < 3; ++i) x[i] = P.num(g[i], 1), lo[i] = P.num(l[i], 0), hi[i] = P.num(u[i], 1);
        cfg.rho_begin = 0.0001;
        cfg.rho_end = 1e-8;
    }
    OptState st{nonstat};
    mra_opt_result res{};
    const mra_status s = mra_opt_minimize(3, x, lo, hi, &cfg, objective, &st, &res);
    if (s != MRA_OK) {
        std::cout << "The optimal parameter values have not been found. Reason: " << mra_last_error() << std::endl;
        return;
    }
    const double ll = -0.5 * (res.f_best + (double)S.st.n_obs() * std::log(2 * 3.14159265359));
    if (nonstat)
        std::cout << "The optimal parameter values are, sigmasq multiplication: " << x[0]
                  << ", beta multiplication: " << x[1] << ", tausq multiplication: " << x[2]
                  << "; The maximum log likelihood is " << ll << ".\n";
    else
        std::cout << "The optimal parameter values are, sigmasq: " << x[0] << ", beta: " << x[1] << ", tausq: " << x[2]
                  << "; The maximum log likelihood is " << ll << ".\n";
}

}  // namespace

void get_optimal_parameters() { run_optimization(false); }
void get_optimal_nonstationary_parameters() { run_optimization(true); }
