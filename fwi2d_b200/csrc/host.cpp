// host.cpp — see host.hpp.  Built with -ffp-contract=off so that every float
// expression rounds exactly as written (indices, b1d, Ricker samples).
#include "host.hpp"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "../../include/fwi2d.h"
#include "detmath.h"

namespace fwi {

// ---------------------------------------------------------------- parameters
bool find_parameter(const std::string& text, const std::string& key, std::string* value) {
    std::istringstream in(text);
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#' || line[0] == ' ') continue;
        if (line.compare(0, key.size(), key) != 0) continue;
        // value starts two characters after '=' (or at 1 when '=' is absent,
        // which is where npos + 2 lands in the reference)
        size_t eq = line.find('=');
        size_t start = (eq == std::string::npos) ? 1 : eq + 2;
        std::string v;
        for (size_t i = start; i < line.size(); ++i) {
            if (line[i] == '#') break;
            v += line[i];
        }
        // A leading quote or bracket is squeezed out the way std::remove without
        // erase leaves it: the kept characters shift left, the tail stays.
        auto squeeze = [](std::string& s, char c) {
            size_t w = 0;
            for (size_t r = 0; r < s.size(); ++r) if (s[r] != c) s[w++] = s[r];
        };
        if (!v.empty() && v[0] == '"') squeeze(v, '"');
        else if (!v.empty() && v[0] == '[') { squeeze(v, '['); squeeze(v, ']'); }
        v.erase(std::remove(v.begin(), v.end(), ' '), v.end());
        *value = v;
        return true;
    }
    return false;
}

ParamFile::ParamFile(const std::string& path) : path_(path) {
    std::ifstream f(path);
    if (!f.is_open()) throw Error(FWI_ERR_IO, "parameters file " + path + " could not be opened");
    std::stringstream ss;
    ss << f.rdbuf();
    text_ = ss.str();
}

bool ParamFile::has(const std::string& key) const {
    std::string v;
    return find_parameter(text_, key, &v) && !v.empty();
}

std::string ParamFile::str(const std::string& key) const {
    std::string v;
    if (!find_parameter(text_, key, &v) || v.empty())
        throw Error(FWI_ERR_PARAM, "missing key '" + key + "' in " + path_);
    return v;
}

int ParamFile::i(const std::string& key) const {
    std::string v = str(key);
    try { return std::stoi(v); }
    catch (...) { throw Error(FWI_ERR_PARAM, "key '" + key + "' is not an integer: '" + v + "'"); }
}

float ParamFile::f(const std::string& key) const {
    std::string v = str(key);
    try { return std::stof(v); }
    catch (...) { throw Error(FWI_ERR_PARAM, "key '" + key + "' is not a number: '" + v + "'"); }
}

std::string ParamFile::str_or(const std::string& key, const std::string& d) const { return has(key) ? str(key) : d; }
float ParamFile::f_or(const std::string& key, float d) const { return has(key) ? f(key) : d; }
int ParamFile::i_or(const std::string& key, int d) const { return has(key) ? i(key) : d; }
uint64_t ParamFile::u64_or(const std::string& key, uint64_t d) const {
    if (!has(key)) return d;
    std::string v = str(key);
    try { return std::stoull(v); }
    catch (...) { throw Error(FWI_ERR_PARAM, "key '" + key + "' is not an unsigned integer: '" + v + "'"); }
}
bool ParamFile::bool_or(const std::string& key, bool d) const {
    if (!has(key)) return d;
    std::string v = str(key);
    std::transform(v.begin(), v.end(), v.begin(), ::tolower);
    if (v == "true" || v == "1" || v == "yes") return true;
    if (v == "false" || v == "0" || v == "no") return false;
    throw Error(FWI_ERR_PARAM, "key '" + key + "' is not a boolean: '" + v + "'");
}

// --------------------------------------------------------------------- files
void read_floats(const std::string& path, float* dst, size_t n) {
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f.is_open()) throw Error(FWI_ERR_IO, path + " could not be opened");
    f.read(reinterpret_cast<char*>(dst), (std::streamsize)(n * sizeof(float)));
    if ((size_t)f.gcount() != n * sizeof(float))
        throw Error(FWI_ERR_IO, path + ": expected " + std::to_string(n) + " float32 values, file is shorter");
}

std::vector<float> read_text_floats(const std::string& path) {
    std::vector<float> v;
    for (std::string line : read_text_lines(path)) {
        std::replace(line.begin(), line.end(), ',', ' ');
        std::istringstream in(line);
        std::string tok;
        while (in >> tok) {
            char* end = nullptr;
            const float x = std::strtof(tok.c_str(), &end);
            if (!end || *end != '\0') throw Error(FWI_ERR_PARAM, path + ": '" + tok + "' is not a number");
            v.push_back(x);
        }
    }
    return v;
}

std::vector<Window> aperture_windows(const Geometry& geo, int nx, float dh, const std::vector<float>& max_offset) {
    const int ns = geo.nsrc();
    std::vector<Window> win(ns, Window{0, nx});
    if (max_offset.empty()) return win;
    if ((int)max_offset.size() != ns)
        throw Error(FWI_ERR_PARAM, "max offsets: " + std::to_string(max_offset.size()) + " values for " +
                                       std::to_string(ns) + " shots");
    for (int s = 0; s < ns; ++s) {
        const double off = max_offset[s], xs = geo.xsrc[s];
        if (!(off > 0)) throw Error(FWI_ERR_PARAM, "max offset of shot " + std::to_string(s + 1) + " must be positive");
        int c0 = (int)std::floor((xs - off) / (double)dh);
        int c1 = (int)std::ceil((xs + off) / (double)dh);
        c0 = std::min(std::max(c0, 0), nx - 1);
        c1 = std::min(std::max(c1, 0), nx - 1);
        while (c1 - c0 + 1 < 9) {
            if (c0 > 0) --c0;
            if (c1 - c0 + 1 < 9 && c1 < nx - 1) ++c1;
        }
        win[s] = Window{c0, c1 - c0 + 1};
    }
    return win;
}

void write_floats(const std::string& path, const float* src, size_t n) {
    std::ofstream f(path, std::ios::out | std::ios::binary);
    if (!f.is_open()) throw Error(FWI_ERR_IO, path + " could not be opened for writing");
    f.write(reinterpret_cast<const char*>(src), (std::streamsize)(n * sizeof(float)));
    if (!f) throw Error(FWI_ERR_IO, "write to " + path + " failed");
}

std::vector<std::string> read_text_lines(const std::string& path) {
    std::ifstream f(path);
    if (!f.is_open()) throw Error(FWI_ERR_IO, path + " could not be opened");
    std::vector<std::string> out;
    std::string line;
    while (std::getline(f, line)) {
        if (!line.empty() && line[0] == '#') continue;
        // blank lines end the reference with an out-of-range split(); skip them
        if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
        out.push_back(line);
    }
    return out;
}

// ------------------------------------------------------------------ geometry
static void parse_xz(const std::vector<std::string>& lines, const std::string& what,
                     std::vector<float>* xs, std::vector<float>* zs) {
    for (const auto& ln : lines) {
        std::vector<std::string> tok;
        std::istringstream ts(ln);
        std::string t;
        while (std::getline(ts, t, ',')) tok.push_back(t);
        if (tok.size() < 2) throw Error(FWI_ERR_PARAM, what + ": line '" + ln + "' is not 'x,z'");
        try {
            xs->push_back(std::stof(tok[0]));
            zs->push_back(std::stof(tok[1]));
        } catch (...) {
            throw Error(FWI_ERR_PARAM, what + ": line '" + ln + "' is not 'x,z'");
        }
    }
}

Geometry read_geometry(const std::string& sps_path, const std::string& rps_path) {
    Geometry g;
    parse_xz(read_text_lines(sps_path), "SPS " + sps_path, &g.xsrc, &g.zsrc);
    parse_xz(read_text_lines(rps_path), "RPS " + rps_path, &g.xrec, &g.zrec);
    if (g.xsrc.empty()) throw Error(FWI_ERR_PARAM, "SPS file " + sps_path + " holds no source");
    if (g.xrec.empty()) throw Error(FWI_ERR_PARAM, "RPS file " + rps_path + " holds no receiver");
    return g;
}

// ------------------------------------------------------------------- wavelet
std::vector<float> make_wavelet(int nt, float dt, float fmax, int* tlag) {
    if (nt <= 0) throw Error(FWI_ERR_PARAM, "time_samples must be positive");
    // Ricker samples in float, as modeling.cu:36-49 computes them.
    float t0 = 2.0f * sqrtf((float)M_PI) / fmax;
    float fc = fmax / (3.0f * sqrtf((float)M_PI));
    *tlag = (int)(t0 / dt) + 1;
    std::vector<double> x(nt);
    for (int n = 0; n < nt; ++n) {
        float td = n * dt - t0;
        float arg = M_PI * M_PI * M_PI * fc * fc * td * td;   // M_PI is double: evaluated in double
        x[n] = (double)(1e5f * (1.0f - 2.0f * arg) * expf(-arg));
    }
    // Half-derivative filter in the frequency domain.  A direct real DFT in
    // double (O(nt^2), once per context) replaces FFTW: bins 0..nt/2 are formed,
    // multiplied by sqrt(i*2*pi*f) and brought back by the Hermitian inverse,
    // which is what an r2c / c2r pair computes.
    const int nh = nt / 2;
    std::vector<double> cs(nt), sn(nt);
    for (int k = 0; k < nt; ++k) {
        double a = 2.0 * M_PI * (double)k / (double)nt;
        cs[k] = std::cos(a);
        sn[k] = std::sin(a);
    }
    std::vector<std::complex<double>> X(nh + 1);
    for (int k = 0; k <= nh; ++k) {
        double re = 0.0, im = 0.0;
        long long idx = 0;
        for (int n = 0; n < nt; ++n) {
            re += x[n] * cs[idx];
            im -= x[n] * sn[idx];
            idx += k;
            if (idx >= nt) idx -= nt;
        }
        double df = 1.0 / (double)(nt * dt);                  // nt*dt is a float product
        double f = k * df;
        std::complex<double> H = std::pow(std::complex<double>(0.0, 2.0 * M_PI * f), 0.5);
        X[k] = std::complex<double>(re, im) * H;
    }
    std::vector<float> w(nt);
    for (int n = 0; n < nt; ++n) {
        double acc = X[0].real();
        long long idx = 0;
        for (int k = 1; k <= nh; ++k) {
            idx += n;
            if (idx >= nt) idx %= nt;
            double term = X[k].real() * cs[idx] - X[k].imag() * sn[idx];
            if (2 * k == nt) acc += X[k].real() * cs[idx];   // Nyquist bin of an even length
            else acc += 2.0 * term;
        }
        w[n] = (float)acc / nt;
    }
    return w;
}

// ------------------------------------------------------------------- damping
int boundary_cells(float length, float dh) { return (int)(length / dh) + 1; }

std::vector<float> make_b1d(int nb, float abc_factor) {
    std::vector<float> b(nb);
    for (int i = 0; i < nb; ++i) b[i] = expf(-powf(abc_factor * (nb - i), 2.0f));
    return b;
}

// ----------------------------------------------------------- random boundary
namespace {
struct Stream {
    uint64_t key, ctr = 0;
    Stream(uint64_t seed, uint32_t shot, uint32_t id) : key(detm::stream_key(seed, shot, id)) {}
    uint64_t next() { return detm::draw(key, ctr++); }
    float uniform(float a, float b) { return a + (b - a) * detm::u01f(next()); }
};
}  // namespace

std::vector<PdsPoint> poisson_disk(float x_max, float z_max, float radius, uint64_t seed, uint32_t shot) {
    Stream rng(seed, shot, detm::STREAM_PDS);
    const float cell = radius / std::sqrt(2.0f);
    const int gx_n = (int)std::ceil(x_max / cell);
    const int gz_n = (int)std::ceil(z_max / cell);
    std::vector<PdsPoint> points, active;
    std::vector<PdsPoint> grid((size_t)gx_n * gz_n, PdsPoint{-1.0f, -1.0f});
    auto insert = [&](const PdsPoint& p) {
        int gx = (int)(p.x / cell), gz = (int)(p.z / cell);
        grid[(size_t)gz + (size_t)gx * gz_n] = p;
    };
    auto valid = [&](const PdsPoint& p) {
        if (p.x < 0 || p.z < 0 || p.x >= x_max || p.z >= z_max) return false;
        int gx = (int)(p.x / cell), gz = (int)(p.z / cell);
        for (int di = -1; di <= 1; ++di)
            for (int dj = -1; dj <= 1; ++dj) {
                int nx = gx + dj, nz = gz + di;
                if (nx >= 0 && nz >= 0 && nx < gx_n && nz < gz_n) {
                    const PdsPoint& q = grid[(size_t)nz + (size_t)nx * gz_n];
                    float dx = q.x - p.x, dz = q.z - p.z;
                    if (q.x != -1.0f && std::sqrt(dx * dx + dz * dz) < radius) return false;
                }
            }
        return true;
    };
    const float two_pi = (float)(2.0 * M_PI);
    PdsPoint p0;
    p0.x = rng.uniform(0.0f, x_max);
    p0.z = rng.uniform(0.0f, z_max);
    points.push_back(p0);
    active.push_back(p0);
    insert(p0);
    while (!active.empty()) {
        size_t idx = (size_t)((rng.next() >> 11) % (uint64_t)active.size());
        PdsPoint base = active[idx];
        bool found = false;
        for (int t = 0; t < 30; ++t) {
            float ang = rng.uniform(0.0f, two_pi);
            float r = rng.uniform(radius, 2.0f * radius);
            PdsPoint q{base.x + r * std::cos(ang), base.z + r * std::sin(ang)};
            if (valid(q)) {
                points.push_back(q);
                active.push_back(q);
                insert(q);
                found = true;
            }
        }
        if (!found) active.erase(active.begin() + (long)idx);
    }
    return points;
}

std::vector<Bump> make_bumps(int nxx, int nzz, int nb, float dh, float ratio, float varVp,
                             uint64_t seed, uint32_t shot) {
    float x_max = (nxx - 1) * dh;
    float z_max = (nzz - 1) * dh;
    std::vector<PdsPoint> pts = poisson_disk(x_max, z_max, ratio, seed, shot);
    float fnb = (float)nb * dh;
    Stream rng(seed, shot, detm::STREAM_BUMP);
    std::vector<Bump> out;
    for (const auto& p : pts) {
        if ((p.x > 0.5f * fnb) && (p.x < x_max - 0.5f * fnb) && (p.z > 0.5f * fnb) && (p.z < z_max - 0.5f * fnb))
            continue;
        Bump b;
        b.xc = p.x;
        b.zc = p.z;
        b.r = rng.uniform(0.2f * ratio, ratio);
        b.A = rng.uniform(0.5f * varVp, varVp);
        b.factor = (rng.next() % 3 == 0) ? 1.0f : -1.0f;
        out.push_back(b);
    }
    return out;
}

// --------------------------------------------------------------- file names
std::string seismogram_name(const std::string& folder, int nt, int nrec, float dt, int shot1) {
    return folder + "seismogram_nt" + std::to_string(nt) + "_nr" + std::to_string(nrec) + "_" +
           std::to_string(int(1e6f * dt)) + "us_shot_" + std::to_string(shot1) + ".bin";
}
std::string rtm_name(const std::string& folder, float fmax, int nz, int nx, float dh) {
    return folder + "RTM_section_" + std::to_string(int(fmax)) + "Hz_" + std::to_string(nz) + "x" +
           std::to_string(nx) + "_" + std::to_string((int)(dh)) + "m.bin";
}
std::string fwi_model_name(const std::string& folder, int iteration, float fmax, int nz, int nx, float dh) {
    return folder + "model_FWI_iteration_" + std::to_string(iteration) + "_" + std::to_string(int(fmax)) + "Hz_" +
           std::to_string(nz) + "x" + std::to_string(nx) + "_" + std::to_string((int)(dh)) + "m.bin";
}
std::string fwi_final_name(const std::string& folder, float fmax, int nz, int nx, float dh) {
    return folder + "final_model_FWI_" + std::to_string(int(fmax)) + "Hz_" + std::to_string(nz) + "x" +
           std::to_string(nx) + "_" + std::to_string((int)(dh)) + "m.bin";
}
std::string convergence_name(const std::string& folder, int max_iteration) {
    return folder + "convergence_" + std::to_string(max_iteration) + "_iterations.txt";
}

}  // namespace fwi
