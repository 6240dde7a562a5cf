// sc_fieldmap.cpp -- 1D field maps in ASTRA format.  Magnetostatic maps as OPAL's
// Astra1DMagnetoStatic reads them (src/Classic/Fields/Astra1DMagnetoStatic.cpp:
// constructor :15-77, readMap :83-160): a header "AstraMagnetostatic
// <accuracy> [TRUE|FALSE]" and lines "z Bz(z)" ('#' comments and blank lines
// skipped, points whose z does not increase by more than 1e-10 dropped).  The
// on-axis field is resampled on an equidistant grid by a natural cubic spline,
// mirrored to an even periodic sequence of 2N points and expanded in a
// Fourier series; the first 2 accuracy - 1 coefficients, normalised to the
// largest |Bz| unless the header says FALSE, are what the device evaluates.
//
// Dynamic (RF standing-wave) maps, as Astra1DDynamic reads them
// (src/Classic/Fields/Astra1DDynamic.cpp: constructor :19-90, readMap
// :96-185): a header "AstraDynamic <accuracy> [TRUE|FALSE]", a line with the
// frequency in MHz, then lines "z Ez(z)"; the same resampling, mirroring and
// series, normalised to the largest |Ez| and scaled by 1e6 (MV/m to V/m).
//
// 2D maps on an (r, z) grid: see read_map2d; 3D maps of RF cavities: see
// read_map3d.
//
// Host C++ only (no CUDA); the evaluation is in sc_common.cuh.
#include <cctype>
#include <cmath>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "scgpu.h"

namespace {

// One content line: '#' starts a comment; lines without a character of the
// reference's set (letters, digits, ". - +" and the byte 0x89) are skipped;
// the line is cut to its first and last such character (Fieldmap::getLine,
// Fieldmap.cpp:519-541, alpha_numeric :802), so a leading sign stays.
bool map_char(unsigned char ch) { return std::isalnum(ch) || ch == '.' || ch == '-' || ch == '+' || ch == 0x89; }

bool content_line(std::ifstream& in, std::string& out) {
    std::string line;
    while (std::getline(in, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.erase(hash);
        size_t first = std::string::npos, last = std::string::npos;
        for (size_t i = 0; i < line.size(); ++i)
            if (map_char((unsigned char)line[i])) {
                if (first == std::string::npos) first = i;
                last = i;
            }
        if (first == std::string::npos) continue;
        out = line.substr(first, last - first + 1);
        return true;
    }
    return false;
}

// A data line holds exactly two numbers (Fieldmap::interpreteLine<double, double>).
bool two_numbers(const std::string& s, double& a, double& b) {
    std::istringstream is(s);
    if (!(is >> a >> b)) return false;
    std::string rest;
    return !(is >> rest);
}

// Natural cubic spline through (x, y) evaluated at t (the second derivatives
// from the tridiagonal system with zero end curvature, then the cubic of the
// interval holding t).
struct NaturalSpline {
    std::vector<double> x, y, m;
    NaturalSpline(const std::vector<double>& xs, const std::vector<double>& ys) : x(xs), y(ys), m(xs.size(), 0.0) {
        const size_t n = x.size();
        if (n < 3) return;
        std::vector<double> c(n, 0.0), d(n, 0.0);
        for (size_t i = 1; i + 1 < n; ++i) {
            const double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
            const double a = h0, bdiag = 2.0 * (h0 + h1), cc = h1;
            const double r = 6.0 * ((y[i + 1] - y[i]) / h1 - (y[i] - y[i - 1]) / h0);
            const double denom = bdiag - a * c[i - 1];
            c[i] = cc / denom;
            d[i] = (r - a * d[i - 1]) / denom;
        }
        for (size_t i = n - 2; i >= 1; --i) {
            m[i] = d[i] - c[i] * m[i + 1];
            if (i == 1) break;
        }
    }
    double operator()(double t) const {
        const size_t n = x.size();
        size_t i = 0;
        if (t >= x[n - 1]) {
            i = n - 2;
        } else {
            size_t lo = 0, hi = n - 1;
            while (hi - lo > 1) {
                const size_t mid = (lo + hi) / 2;
                if (x[mid] > t)
                    hi = mid;
                else
                    lo = mid;
            }
            i = lo;
        }
        const double h = x[i + 1] - x[i];
        const double A = (x[i + 1] - t) / h, B = (t - x[i]) / h;
        return A * y[i] + B * y[i + 1] + ((A * A * A - A) * m[i] + (B * B * B - B) * m[i + 1]) * h * h / 6.0;
    }
};

// Reads a magnetostatic ("AstraM...") or, with dynamic, a dynamic
// ("AstraD...") map; the dynamic header line is followed by the frequency in
// MHz (Astra1DDynamic.cpp:19-90) and its coefficients carry the factor 1e6
// of the MV/m -> V/m conversion (:150-153).
int read_astra1d(const char* path, bool dynamic, double* coefs, int max_coefs, int* ncoefs, double* zbegin,
                 double* zend, double* period, double* freq_mhz) {
    if (!path || !coefs || !ncoefs || !zbegin || !zend || !period) return SCGPU_ERR_ARG;
    std::ifstream in(path);
    if (!in) return SCGPU_ERR_ARG;
    std::string line;
    if (!content_line(in, line)) return SCGPU_ERR_ARG;
    std::istringstream hs(line);
    std::string name, flag;
    int accuracy = 0;
    if (!(hs >> name >> accuracy) || name.compare(0, 6, dynamic ? "AstraD" : "AstraM") != 0 || accuracy < 1)
        return SCGPU_ERR_ARG;
    bool normalize = true;
    if (hs >> flag) {
        for (char& ch : flag) ch = (char)std::toupper((unsigned char)ch);
        if (flag != "TRUE" && flag != "FALSE") return SCGPU_ERR_ARG;
        normalize = flag == "TRUE";
    }
    if (dynamic) {
        if (!content_line(in, line)) return SCGPU_ERR_ARG;
        std::istringstream fs(line);
        double f = 0.0;
        std::string rest;
        if (!(fs >> f) || (fs >> rest) || !(f > 0.0)) return SCGPU_ERR_ARG;
        if (freq_mhz) *freq_mhz = f;
    }
    std::vector<double> zs, bz;
    double z = 0.0, b = 0.0, last = 0.0, zlast = 0.0;
    while (content_line(in, line)) {
        if (!two_numbers(line, z, b)) return SCGPU_ERR_ARG;
        zlast = z;  // the last line read sets zend, accepted or not (:45-52)
        if (zs.empty() || z - last > 1e-10) {
            zs.push_back(z);
            bz.push_back(b);
            last = z;
        }
    }
    const int N = (int)zs.size();
    if (N < 3 || 2 * accuracy - 1 > max_coefs || accuracy > N) return SCGPU_ERR_ARG;
    const double zb = zs[0], ze = zlast;
    const double dz = (ze - zb) / (N - 1);
    double bmax = 0.0;
    for (double v : bz) bmax = std::fmax(bmax, std::fabs(v));
    if (!normalize) bmax = 1.0;
    if (!(bmax > 0.0)) return SCGPU_ERR_ARG;
    // equidistant resampling, then the mirror image in front: 2N samples
    const NaturalSpline spline(zs, bz);
    std::vector<double> seq(2 * (size_t)N);
    for (int i = 0; i < N - 1; ++i) seq[N + i] = spline(zb + dz * i);
    seq[2 * (size_t)N - 1] = bz[N - 1];
    for (int i = 0; i < N; ++i) seq[i] = seq[2 * (size_t)N - 1 - i];
    // forward DFT X_k = sum_j x_j exp(-2 pi i j k / 2N) for k < accuracy, in long double
    const long n = 2L * N;
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < accuracy; ++k) {
        long double re = 0.0L, im = 0.0L;
        for (long j = 0; j < n; ++j) {
            const long double a = two_pi * (long double)((j * (long)k) % n) / (long double)n;
            re += (long double)seq[j] * cosl(a);
            im -= (long double)seq[j] * sinl(a);
        }
        const double u = dynamic ? 1.0e6 : 1.0;
        if (k == 0) {
            coefs[0] = u * (double)re / (bmax * 2. * N);
        } else {
            coefs[2 * k - 1] = u * (double)re / (bmax * N);
            coefs[2 * k] = u * (double)im / (bmax * N);
        }
    }
    *ncoefs = 2 * accuracy - 1;
    *zbegin = zb;
    *zend = ze;
    *period = 2.0 * N * (ze - zb) / (N - 1);
    return SCGPU_OK;
}

// 2D maps on an (r, z) grid, as FM2DMagnetoStatic and FM2DDynamic read them
// (src/Classic/Fields/FM2DMagnetoStatic.cpp: constructor :14-95, readMap
// :101-155; FM2DDynamic.cpp: constructor :15-104, readMap :110-170): a header
// "2DMagnetoStatic XZ|ZX [TRUE|FALSE]" or "2DDynamic XZ|ZX [TRUE|FALSE]";
// for XZ the lines "zbegin zend nz", (dynamic: the frequency in MHz),
// "rbegin rend nr" in cm and intervals, then (nz+1)(nr+1) value lines, r
// outer and z inner: "Bz Br" or "Ez Er - Ht"; for ZX the r line first and
// z outer, "Br Bz" or "Er Ez Ht -".  Lengths become m, counts become grid
// points; unless FALSE the values are divided by the largest |Bz| (|Ez|) on
// the axis; a dynamic map's E goes from MV/m to V/m (x 1e6 / Ezmax) and its
// H to B (x mu_0 / Ezmax, mu_0 = 1.256637061e-06 as Physics.h:55).
// values: component c at grid point (z i, r j) at values[(c nr + j) nz + i],
// components Bz, Br or Ez, Er, Bt.
struct Map2D {
    bool dynamic = false;
    int nz = 0, nr = 0;  // grid points
    double zbegin = 0, zend = 0, rbegin = 0, rend = 0, freq_mhz = 0;
    std::vector<double> v;
};

bool numbers(const std::string& s, double* out, int n) {
    std::istringstream is(s);
    for (int k = 0; k < n; ++k)
        if (!(is >> out[k])) return false;
    std::string rest;
    return !(is >> rest);
}

bool range_line(std::ifstream& in, double& a, double& b, int& n) {
    std::string line;
    if (!content_line(in, line)) return false;
    std::istringstream is(line);
    std::string rest;
    if (!(is >> a >> b >> n) || (is >> rest)) return false;
    return n >= 1 && n <= (1 << 26);  // interval counts; the grid sizes are checked by the callers
}

int read_map2d(const char* path, Map2D& m) {
    if (!path) return SCGPU_ERR_ARG;
    std::ifstream in(path);
    if (!in) return SCGPU_ERR_ARG;
    std::string line;
    if (!content_line(in, line)) return SCGPU_ERR_ARG;
    std::istringstream hs(line);
    std::string name, orient, flag;
    if (!(hs >> name >> orient)) return SCGPU_ERR_ARG;
    if (name.compare(0, 4, "2DMa") == 0)
        m.dynamic = false;
    else if (name.compare(0, 4, "2DDy") == 0)
        m.dynamic = true;
    else
        return SCGPU_ERR_ARG;
    bool normalize = true;
    if (hs >> flag) {
        for (char& ch : flag) ch = (char)std::toupper((unsigned char)ch);
        if (flag != "TRUE" && flag != "FALSE") return SCGPU_ERR_ARG;
        normalize = flag == "TRUE";
    }
    const bool swap = orient == "ZX";
    if (!swap && orient != "XZ") return SCGPU_ERR_ARG;
    int nzi = 0, nri = 0;
    auto freq = [&]() {
        if (!m.dynamic) return true;
        if (!content_line(in, line)) return false;
        double f = 0.0;
        return numbers(line, &f, 1) && (m.freq_mhz = f, true);
    };
    if (swap) {
        if (!range_line(in, m.rbegin, m.rend, nri) || !freq() || !range_line(in, m.zbegin, m.zend, nzi))
            return SCGPU_ERR_ARG;
    } else {
        if (!range_line(in, m.zbegin, m.zend, nzi) || !freq() || !range_line(in, m.rbegin, m.rend, nri))
            return SCGPU_ERR_ARG;
    }
    m.nz = nzi + 1;
    m.nr = nri + 1;
    const int nc = m.dynamic ? 3 : 2;
    const size_t np = (size_t)m.nz * m.nr;
    if (np > ((size_t)1 << 26)) return SCGPU_ERR_ARG;
    m.v.assign(nc * np, 0.0);
    double* A = m.v.data();  // Bz or Ez
    double* B = A + np;      // Br or Er
    double* T = A + 2 * np;  // Bt (dynamic)
    double x[4];
    const int per = m.dynamic ? 4 : 2;
    for (size_t k = 0; k < np; ++k) {
        if (!content_line(in, line) || !numbers(line, x, per)) return SCGPU_ERR_ARG;
        size_t i, j;  // z, r
        if (swap) {
            i = k / m.nr;
            j = k % m.nr;
        } else {
            j = k / m.nz;
            i = k % m.nz;
        }
        const size_t at = i + j * m.nz;
        if (swap) {
            B[at] = x[0];
            A[at] = x[1];
            if (m.dynamic) T[at] = x[2];
        } else {
            A[at] = x[0];
            B[at] = x[1];
            if (m.dynamic) T[at] = x[3];
        }
    }
    if (content_line(in, line)) return SCGPU_ERR_ARG;  // interpreteEOF: nothing after the values
    m.rbegin /= 100.0;
    m.rend /= 100.0;
    m.zbegin /= 100.0;
    m.zend /= 100.0;
    double amax = 0.0;
    if (normalize) {
        for (int i = 0; i < m.nz; ++i)
            if (std::abs(A[i]) > amax) amax = std::abs(A[i]);
        if (!(amax > 0.0)) return SCGPU_ERR_ARG;
    } else {
        amax = 1.0;
    }
    if (m.dynamic) {
        const double mu_0 = 1.256637061e-06;
        for (size_t k = 0; k < np; ++k) {
            A[k] *= 1.e6 / amax;
            B[k] *= 1.e6 / amax;
            T[k] *= mu_0 / amax;
        }
    } else if (normalize) {
        for (size_t k = 0; k < np; ++k) {
            A[k] /= amax;
            B[k] /= amax;
        }
    }
    return SCGPU_OK;
}

// 3D maps of RF cavities, as FM3DDynamic reads them
// (src/Classic/Fields/FM3DDynamic.cpp: constructor :17-107, readMap
// :113-220): a header "3DDynamic [TRUE|FALSE]", the frequency in MHz, the
// lines "xbegin xend nx", "ybegin yend ny", "zbegin zend nz" in cm and
// intervals, then (nx+1)(ny+1)(nz+1) lines "Ex Ey Ez Hx Hy Hz" [MV/m, A/m],
// x outer, y, z inner.  Lengths become m, counts grid points; unless FALSE
// the values are divided by the largest |Ez| on the grid line along z
// nearest the axis (the x index ceil(-xbegin / hx), one less when that grid
// x exceeds 0.5, likewise y); E is scaled by 1e6 / Ezmax (MV/m to V/m) and H
// by mu_0 / Ezmax (to B).  values: component c (Ex, Ey, Ez, Bx, By, Bz) at
// (x i, y j, z k) at values[c nx ny nz + (i ny + j) nz + k].
struct Map3D {
    int nx = 0, ny = 0, nz = 0;  // grid points
    double xbegin = 0, xend = 0, ybegin = 0, yend = 0, zbegin = 0, zend = 0, freq_mhz = 0;
    std::vector<double> v;
};

int read_map3d(const char* path, Map3D& m) {
    if (!path) return SCGPU_ERR_ARG;
    std::ifstream in(path);
    if (!in) return SCGPU_ERR_ARG;
    std::string line;
    if (!content_line(in, line)) return SCGPU_ERR_ARG;
    std::istringstream hs(line);
    std::string name, flag, rest;
    if (!(hs >> name) || name.compare(0, 4, "3DDy") != 0) return SCGPU_ERR_ARG;
    bool normalize = true;
    if (hs >> flag) {
        for (char& ch : flag) ch = (char)std::toupper((unsigned char)ch);
        if (flag != "TRUE" && flag != "FALSE") return SCGPU_ERR_ARG;
        normalize = flag == "TRUE";
        if (hs >> rest) return SCGPU_ERR_ARG;
    }
    int nxi = 0, nyi = 0, nzi = 0;
    if (!content_line(in, line) || !numbers(line, &m.freq_mhz, 1)) return SCGPU_ERR_ARG;
    if (!range_line(in, m.xbegin, m.xend, nxi) || !range_line(in, m.ybegin, m.yend, nyi) ||
        !range_line(in, m.zbegin, m.zend, nzi))
        return SCGPU_ERR_ARG;
    m.nx = nxi + 1;
    m.ny = nyi + 1;
    m.nz = nzi + 1;
    const size_t np = (size_t)m.nx * m.ny * m.nz;
    if ((size_t)m.nx * m.ny > ((size_t)1 << 26) || np > ((size_t)1 << 26)) return SCGPU_ERR_ARG;
    m.v.assign(6 * np, 0.0);
    double x[6];
    for (size_t k = 0; k < np; ++k) {  // (i ny + j) nz + k in file order
        if (!content_line(in, line) || !numbers(line, x, 6)) return SCGPU_ERR_ARG;
        for (int c = 0; c < 6; ++c) m.v[c * np + k] = x[c];
    }
    if (content_line(in, line)) return SCGPU_ERR_ARG;  // interpreteEOF: nothing after the values
    m.xbegin /= 100.0;
    m.xend /= 100.0;
    m.ybegin /= 100.0;
    m.yend /= 100.0;
    m.zbegin /= 100.0;
    m.zend /= 100.0;
    const double hx = (m.xend - m.xbegin) / nxi, hy = (m.yend - m.ybegin) / nyi;
    double ezmax = 1.0;
    if (normalize) {
        int ix = (int)std::ceil(-m.xbegin / hx);
        if (ix * hx + m.xbegin > 0.5) --ix;
        int iy = (int)std::ceil(-m.ybegin / hy);
        if (iy * hy + m.ybegin > 0.5) --iy;
        // a map whose axis line lies outside the grid has no reference value
        if (ix < 0 || ix >= m.nx || iy < 0 || iy >= m.ny) return SCGPU_ERR_ARG;
        const double* ez = m.v.data() + 2 * np + ((size_t)ix * m.ny + iy) * m.nz;
        ezmax = 0.0;
        for (int k = 0; k < m.nz; ++k)
            if (std::abs(ez[k]) > ezmax) ezmax = std::abs(ez[k]);
        if (!(ezmax > 0.0)) return SCGPU_ERR_ARG;
    }
    const double mu_0 = 1.256637061e-06;
    for (size_t k = 0; k < 3 * np; ++k) m.v[k] *= 1e6 / ezmax;
    for (size_t k = 3 * np; k < 6 * np; ++k) m.v[k] *= mu_0 / ezmax;
    return SCGPU_OK;
}

}  // namespace

namespace sc {
// true when the map file's first word names a 3D dynamic map (3DDynamic);
// a 3D magnetostatic map ("3DMa") answers 2
int fieldmap_kind_3d(const char* path) {
    if (!path) return 0;
    std::ifstream in(path);
    std::string line;
    if (!in || !content_line(in, line)) return 0;
    if (line.compare(0, 4, "3DDy") == 0) return 1;
    if (line.compare(0, 4, "3DMa") == 0) return 2;
    return 0;
}

// the 3D map for the element table (sc_api.cu): grid points {nx, ny, nz},
// ranges {xbegin, xend, ybegin, yend, zbegin, zend} [m], frequency [MHz]
int fieldmap_3d(const char* path, int* n, double* ranges, double* freq_mhz, std::vector<double>* values) {
    Map3D m;
    const int rc = read_map3d(path, m);
    if (rc) return rc;
    n[0] = m.nx;
    n[1] = m.ny;
    n[2] = m.nz;
    const double r[6] = {m.xbegin, m.xend, m.ybegin, m.yend, m.zbegin, m.zend};
    for (int k = 0; k < 6; ++k) ranges[k] = r[k];
    *freq_mhz = m.freq_mhz;
    values->swap(m.v);
    return SCGPU_OK;
}

// the map's type from its first word, as Fieldmap::readHeader does
// (Fieldmap.cpp:296-335, the first four characters)
bool fieldmap_is_2d(const char* path) {
    if (!path) return false;
    std::ifstream in(path);
    std::string line;
    if (!in || !content_line(in, line)) return false;
    return line.compare(0, 4, "2DMa") == 0 || line.compare(0, 4, "2DDy") == 0;
}

// the map for the element table (sc_api.cu)
int fieldmap_2d(const char* path, bool* dynamic, int* nz, int* nr, double* zbegin, double* zend, double* rbegin,
                double* rend, double* freq_mhz, std::vector<double>* values) {
    Map2D m;
    const int rc = read_map2d(path, m);
    if (rc) return rc;
    *dynamic = m.dynamic;
    *nz = m.nz;
    *nr = m.nr;
    *zbegin = m.zbegin;
    *zend = m.zend;
    *rbegin = m.rbegin;
    *rend = m.rend;
    *freq_mhz = m.freq_mhz;
    values->swap(m.v);
    return SCGPU_OK;
}
}  // namespace sc

extern "C" {

int scgpu_fieldmap_2d(const char* path, int* dynamic, int* nz, int* nr, double* ranges, double* frequency_mhz,
                      double* values, long long capacity) {
    if (!path || !dynamic || !nz || !nr || !ranges || !frequency_mhz) return SCGPU_ERR_ARG;
    Map2D m;
    const int rc = read_map2d(path, m);
    if (rc) return rc;
    *dynamic = m.dynamic ? 1 : 0;
    *nz = m.nz;
    *nr = m.nr;
    ranges[0] = m.zbegin;
    ranges[1] = m.zend;
    ranges[2] = m.rbegin;
    ranges[3] = m.rend;
    *frequency_mhz = m.freq_mhz;
    if (values) {
        if (capacity < (long long)m.v.size()) return SCGPU_ERR_ARG;
        for (size_t k = 0; k < m.v.size(); ++k) values[k] = m.v[k];
    }
    return SCGPU_OK;
}

int scgpu_fieldmap_3d(const char* path, int* n, double* ranges, double* frequency_mhz, double* values,
                      long long capacity) {
    if (!path || !n || !ranges || !frequency_mhz) return SCGPU_ERR_ARG;
    std::vector<double> v;
    const int rc = sc::fieldmap_3d(path, n, ranges, frequency_mhz, &v);
    if (rc) return rc;
    if (values) {
        if (capacity < (long long)v.size()) return SCGPU_ERR_ARG;
        for (size_t k = 0; k < v.size(); ++k) values[k] = v[k];
    }
    return SCGPU_OK;
}

int scgpu_fieldmap_astra1d(const char* path, double* coefs, int max_coefs, int* ncoefs, double* zbegin, double* zend,
                           double* period) {
    return read_astra1d(path, false, coefs, max_coefs, ncoefs, zbegin, zend, period, nullptr);
}

int scgpu_fieldmap_astra1d_dynamic(const char* path, double* coefs, int max_coefs, int* ncoefs, double* zbegin,
                                   double* zend, double* period, double* frequency_mhz) {
    if (!frequency_mhz) return SCGPU_ERR_ARG;
    return read_astra1d(path, true, coefs, max_coefs, ncoefs, zbegin, zend, period, frequency_mhz);
}

}  // extern "C"
