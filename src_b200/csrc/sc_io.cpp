// sc_io.cpp -- the reference's file formats on the host side of the C ABI:
//
//   * ASCII particle distributions read by DISTRIBUTION, TYPE=FROMFILE
//     (Distribution::getNumberOfParticlesInFile / createDistributionFromFile,
//     src/Distribution/Distribution.cpp:1074-1159, converteVToBetaGamma :1047-1053);
//   * the SDDS statistics file (.stat) of DataSink (src/Structure/DataSink.cpp:
//     header :585-1032, rows :281-449, stream settings :1330-1334).
//
// Plain C++ (no CUDA): the statistics row itself is computed on the device by
// scgpu_stat_row (sc_api.cu).
#include <cctype>
#include <cerrno>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <sstream>
#include <string>

#include "scgpu.h"

namespace {

// The statistics columns, in file order: name, SDDS type, units, description.
struct StatColumn {
    const char* name;
    const char* type;
    const char* units;
    const char* description;
};

const StatColumn kStatColumns[SCGPU_STAT_COLUMNS] = {
    {"t", "double", "ns", "1 Time"},
    {"s", "double", "m", "2 Average Longitudinal Position"},
    {"numParticles", "long", "1", "3 Number of Macro Particles"},
    {"charge", "double", "1", "4 Bunch Charge"},
    {"energy", "double", "MeV", "5 Mean Energy"},
    {"rms_x", "double", "m", "6 RMS Beamsize in x"},
    {"rms_y", "double", "m", "7 RMS Beamsize in y"},
    {"rms_s", "double", "m", "8 RMS Beamsize in s"},
    {"rms_px", "double", "1", "9 RMS Momenta in x"},
    {"rms_py", "double", "1", "10 RMS Momenta in y"},
    {"rms_ps", "double", "1", "11 RMS Momenta in s"},
    {"emit_x", "double", "m", "12 Normalized Emittance x"},
    {"emit_y", "double", "m", "13 Normalized Emittance y"},
    {"emit_s", "double", "m", "14 Normalized Emittance s"},
    {"mean_x", "double", "m", "15 Mean Beam Position in x"},
    {"mean_y", "double", "m", "16 Mean Beam Position in y"},
    {"mean_s", "double", "m", "17 Mean Beam Position in s"},
    {"ref_x", "double", "m", "18 x coordinate of reference particle in lab cs"},
    {"ref_y", "double", "m", "19 y coordinate of reference particle in lab cs"},
    {"ref_z", "double", "m", "20 z coordinate of reference particle in lab cs"},
    {"ref_px", "double", "1", "21 x momentum of reference particle in lab cs"},
    {"ref_py", "double", "1", "22 y momentum of reference particle in lab cs"},
    {"ref_pz", "double", "1", "23 z momentum of reference particle in lab cs"},
    {"max_x", "double", "m", "24 Max Beamsize in x"},
    {"max_y", "double", "m", "25 Max Beamsize in y"},
    {"max_s", "double", "m", "26 Max Beamsize in s"},
    {"xpx", "double", "1", "27 Correlation xpx"},
    {"ypy", "double", "1", "28 Correlation ypyy"},
    {"zpz", "double", "1", "29 Correlation zpz"},
    {"Dx", "double", "m", "30 Dispersion in x"},
    {"DDx", "double", "1", "31 Derivative of dispersion in x"},
    {"Dy", "double", "m", "32 Dispersion in y"},
    {"DDy", "double", "1", "33 Derivative of dispersion in y"},
    {"Bx_ref", "double", "T", "34 Bx-Field component of ref particle"},
    {"By_ref", "double", "T", "35 By-Field component of ref particle"},
    {"Bz_ref", "double", "T", "36 Bz-Field component of ref particle"},
    {"Ex_ref", "double", "MV/m", "37 Ex-Field component of ref particle"},
    {"Ey_ref", "double", "MV/m", "38 Ey-Field component of ref particle"},
    {"Ez_ref", "double", "MV/m", "39 Ez-Field component of ref particle"},
    {"dE", "double", "MeV", "40 energy spread of the beam"},
    {"dt", "double", "ns", "41 time step size"},
    {"partsOutside", "double", "1", "42 outside n*sigma of the beam"},
    {"R0_x", "double", "m", "43 R0 Particle position in x"},
    {"R0_y", "double", "m", "44 R0 Particle position in y"},
    {"R0_s", "double", "m", "45 R0 Particle position in z"},
    {"P0_x", "double", "1", "46 R0 Particle momentum in x"},
    {"P0_y", "double", "1", "47 R0 Particle momentum in y"},
    {"P0_s", "double", "1", "48 R0 Particle momentum in z"},
};

// Column indices written as integers (size_t values in the reference's row).
bool integer_column(int c) { return c == 2 || c == 41; }

// One value as the reference's stream writes it: precision 15, scientific
// (DataSink::open_m), followed by std::setw(10) << "\t", i.e. nine spaces
// and a tab.
void put_value(std::FILE* f, double v, bool integer) {
    if (integer)
        std::fprintf(f, "%lld         \t", (long long)v);
    else
        std::fprintf(f, "%.15e         \t", v);
}

// FROMFILE's momentum conversion from eV (Distribution.cpp:1047-1053).
double ev_to_beta_gamma(double value_ev, double mass_ev) {
    double value = std::copysign(std::sqrt(std::pow(std::abs(value_ev) / mass_ev + 1.0, 2.0) - 1.0), value_ev);
    if (std::abs(value) < DBL_EPSILON) value = std::copysign(std::sqrt(2 * std::abs(value_ev) / mass_ev), value_ev);
    return value;
}

// The particle-count line: the first line that is not empty once a
// "[[:space:]]*#.*" comment is removed (Distribution.cpp:1084-1098).
bool count_line(std::ifstream& in, long long* n) {
    std::string line;
    do {
        if (!std::getline(in, line)) return false;
        size_t hash = line.find('#');
        if (hash != std::string::npos) {
            size_t start = hash;
            while (start > 0 && std::isspace((unsigned char)line[start - 1])) --start;
            line.erase(start);
        }
    } while (line.empty());
    std::istringstream ls(line);
    long tmp = 0;
    ls >> tmp;
    *n = tmp;
    return true;
}

}  // namespace

extern "C" {

int scgpu_read_fromfile_count(const char* path, long long* n) {
    if (!path || !n) return SCGPU_ERR_ARG;
    std::ifstream in(path);
    if (!in) return SCGPU_ERR_ARG;
    long long cnt = 0;
    if (!count_line(in, &cnt) || cnt <= 0) return SCGPU_ERR_ARG;
    *n = cnt;
    return SCGPU_OK;
}

int scgpu_read_fromfile(const char* path, long long capacity, double* R, double* P, int momenta_in_ev, double mass_ev,
                        long long* n) {
    if (!path || !R || !P || !n) return SCGPU_ERR_ARG;
    if (momenta_in_ev && !(mass_ev > 0.0)) return SCGPU_ERR_ARG;
    std::ifstream in(path);
    if (!in) return SCGPU_ERR_ARG;
    long long cnt = 0;
    if (!count_line(in, &cnt) || cnt <= 0) return SCGPU_ERR_ARG;
    if (cnt > capacity) return SCGPU_ERR_ARG;
    for (long long i = 0; i < cnt; ++i) {
        double* r = R + 3 * i;
        double* p = P + 3 * i;
        // record order x px y py z pz (Distribution.cpp:1152-1157)
        if (!(in >> r[0] >> p[0] >> r[1] >> p[1] >> r[2] >> p[2])) return SCGPU_ERR_ARG;
        if (momenta_in_ev)
            for (int d = 0; d < 3; ++d) p[d] = ev_to_beta_gamma(p[d], mass_ev);
    }
    *n = cnt;
    return SCGPU_OK;
}

int scgpu_write_fromfile(const char* path, long long n, const double* R, const double* P) {
    if (!path || !R || !P || n <= 0) return SCGPU_ERR_ARG;
    std::FILE* f = std::fopen(path, "w");
    if (!f) return SCGPU_ERR_ARG;
    std::fprintf(f, "%lld\n", n);
    for (long long i = 0; i < n; ++i) {
        const double* r = R + 3 * i;
        const double* p = P + 3 * i;
        std::fprintf(f, "%.17g %.17g %.17g %.17g %.17g %.17g\n", r[0], p[0], r[1], p[1], r[2], p[2]);
    }
    return std::fclose(f) == 0 ? SCGPU_OK : SCGPU_ERR_ARG;
}

const char* scgpu_stat_column_name(int column) {
    return (column >= 0 && column < SCGPU_STAT_COLUMNS) ? kStatColumns[column].name : nullptr;
}

int scgpu_sdds_write_header(const char* path, const char* input_name, int processors, const char* revision,
                            const char* flavor) {
    if (!path) return SCGPU_ERR_ARG;
    std::FILE* f = std::fopen(path, "w");
    if (!f) return SCGPU_ERR_ARG;
    char date[32], tod[32];
    const std::time_t now = std::time(nullptr);
    std::tm tmv{};
    localtime_r(&now, &tmv);
    std::strftime(date, sizeof date, "%d/%m/%Y", &tmv);
    std::strftime(tod, sizeof tod, "%H:%M:%S", &tmv);
    const char* ind = "        ";
    std::fprintf(f, "SDDS1\n");
    std::fprintf(f, "&description\n%stext=\"Statistics data '%s' %s %s\",\n%scontents=\"stat parameters\"\n&end\n", ind,
                 input_name ? input_name : "", date, tod, ind);
    std::fprintf(f, "&parameter\n%sname=processors,\n%stype=long,\n%sdescription=\"Number of Cores used\"\n&end\n", ind, ind,
                 ind);
    std::fprintf(f, "&parameter\n%sname=revision,\n%stype=string,\n%sdescription=\"git revision of opal\"\n&end\n", ind, ind,
                 ind);
    std::fprintf(f, "&parameter\n%sname=flavor,\n%stype=string,\n%sdescription=\"OPAL flavor that wrote file\"\n&end\n", ind,
                 ind, ind);
    for (const StatColumn& c : kStatColumns)
        std::fprintf(f, "&column\n%sname=%s,\n%stype=%s,\n%sunits=%s,\n%sdescription=\"%s\"\n&end\n", ind, c.name, ind, c.type,
                     ind, c.units, ind, c.description);
    std::fprintf(f, "&data\n%smode=ascii,\n%sno_row_counts=1\n&end\n", ind, ind);
    std::fprintf(f, "%d\n%s\n%s\n", processors, revision ? revision : "", flavor ? flavor : "opal-t");
    return std::fclose(f) == 0 ? SCGPU_OK : SCGPU_ERR_ARG;
}

int scgpu_sdds_append_row(const char* path, const double* row, int with_particle0) {
    if (!path || !row) return SCGPU_ERR_ARG;
    std::FILE* f = std::fopen(path, "a");
    if (!f) return SCGPU_ERR_ARG;
    // R0 / P0 only from a single-rank run with particles (DataSink.cpp:419-426)
    const int ncol = with_particle0 ? SCGPU_STAT_COLUMNS : SCGPU_STAT_COLUMNS - 6;
    for (int c = 0; c < ncol; ++c) put_value(f, row[c], integer_column(c));
    std::fprintf(f, "\n");
    return std::fclose(f) == 0 ? SCGPU_OK : SCGPU_ERR_ARG;
}

}  // extern "C"
