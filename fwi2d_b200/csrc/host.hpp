// host.hpp — host-side setup of the engine: parameters.txt, geometry, raw
// float32 files, wavelet, damping table, grid indices and the host half of the
// random boundary.  Each routine cites the reference routine it follows.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace fwi {

// Error carrying one of the FWI_ERR_* status codes of fwi2d.h.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// ---- parameters.txt ------------------------------------------------------
// Value of `key` following catch_parameter (src/admin/admin.cpp:53-98): the
// first line that does not start with '#' or ' ' and whose text starts with
// `key`; the value runs from two characters after '=' up to '#', with spaces
// removed.  Returns false when no line matches (the reference returns "" and
// the following std::stoi/stof throws).
bool find_parameter(const std::string& text, const std::string& key, std::string* value);

class ParamFile {
public:
    explicit ParamFile(const std::string& path);
    const std::string& path() const { return path_; }
    bool has(const std::string& key) const;
    std::string str(const std::string& key) const;   // FWI_ERR_PARAM when missing
    int         i(const std::string& key) const;     // std::stoi semantics
    float       f(const std::string& key) const;     // std::stof semantics
    std::string str_or(const std::string& key, const std::string& dflt) const;
    float       f_or(const std::string& key, float dflt) const;
    int         i_or(const std::string& key, int dflt) const;
    uint64_t    u64_or(const std::string& key, uint64_t dflt) const;
    bool        bool_or(const std::string& key, bool dflt) const;
private:
    std::string path_, text_;
};

// ---- files ----------------------------------------------------------------
// import_binary_float / export_binary_float (admin.cpp:13-37).  The read fails
// on a short file instead of leaving the tail untouched.
void read_floats(const std::string& path, float* dst, size_t n);
void write_floats(const std::string& path, const float* src, size_t n);
// import_text_file (admin.cpp:39-51): lines not starting with '#'.
std::vector<std::string> read_text_lines(const std::string& path);

// ---- geometry (src/geometry/geometry.cpp:3-43) -----------------------------
struct Geometry {
    std::vector<float> xsrc, zsrc, xrec, zrec;
    int nsrc() const { return (int)xsrc.size(); }
    int nrec() const { return (int)xrec.size(); }
};
Geometry read_geometry(const std::string& sps_path, const std::string& rps_path);

// ---- aperture windows (batched uneven-aperture surveys) -----------------------
// Not in the reference, which models every shot on the whole model.  Shot s
// is modeled on the model columns [c0, c0 + w): the columns within
// max_offset[s] of its source, c0 = floor((xs - off)/dh), c1 = ceil((xs + off)/dh),
// both clamped to [0, nx); windows narrower than 9 columns are widened about
// the source.  An empty max_offset gives every shot the whole model.
struct Window {
    int c0, w;
};
std::vector<Window> aperture_windows(const Geometry& geo, int nx, float dh, const std::vector<float>& max_offset);
// Whitespace- or comma-separated floats of a text file ('#' lines skipped).
std::vector<float> read_text_floats(const std::string& path);

// ---- wavelet (modeling.cu:32-90) -------------------------------------------
// Ricker of peak fmax/(3 sqrt(pi)) delayed by t0 = 2 sqrt(pi)/fmax, scaled by
// 1e5, filtered by (i 2 pi f)^(1/2) in double precision and divided by nt.
// tlag = int(t0/dt) + 1.
std::vector<float> make_wavelet(int nt, float dt, float fmax, int* tlag);

// ---- damping (modeling.cu:113-150) -----------------------------------------
int boundary_cells(float length, float dh);          // int(length/dh) + 1
std::vector<float> make_b1d(int nb, float abc_factor); // expf(-powf(f*(nb-i),2))

// ---- indices (modeling.cu:252-277) ------------------------------------------
inline int grid_index(float coord, float dh, int nb) { return (int)((coord + 0.5f * dh) / dh) + nb; }

// ---- random boundary, host half (modeling.cu:431-465, admin.cpp:112-206) ----
struct Bump { float xc, zc, r, A, factor; };
// Poisson-disk points over [0,x_max) x [0,z_max) with Bridson's method (30
// tries per active point) driven by the counter-based generator of detmath.h.
struct PdsPoint { float x, z; };
std::vector<PdsPoint> poisson_disk(float x_max, float z_max, float radius, uint64_t seed, uint32_t shot);
// Points outside the inner box shrunk by 0.5*nb*dh, each with radius
// U(0.2 ratio, ratio), amplitude U(0.5 varVp, varVp) and sign + with
// probability 1/3 (rand()%3==0), in sampling order.
std::vector<Bump> make_bumps(int nxx, int nzz, int nb, float dh, float ratio, float varVp,
                             uint64_t seed, uint32_t shot);

// ---- CFL -----------------------------------------------------------------
// The 8th-order Laplacian has symbol magnitude 6.5016/dh^2 per axis at the
// Nyquist wavenumber, so leapfrog stability needs vmax*dt/dh <= 2/sqrt(13.0032).
constexpr double kCflLimit = 0.55463;

// Output file names with the reference's std::to_string formatting.
std::string seismogram_name(const std::string& folder, int nt, int nrec, float dt, int shot1);
std::string rtm_name(const std::string& folder, float fmax, int nz, int nx, float dh);
std::string fwi_model_name(const std::string& folder, int iteration, float fmax, int nz, int nx, float dh);
std::string fwi_final_name(const std::string& folder, float fmax, int nz, int nx, float dh);
std::string convergence_name(const std::string& folder, int max_iteration);

}  // namespace fwi
