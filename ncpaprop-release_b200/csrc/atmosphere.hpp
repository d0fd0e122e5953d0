// Host-side NCPA atmospheric profile reader: the file format and unit
// handling of NCPA::Atmosphere1D (src/atmosphere/Atmosphere1D.cpp:85-285) and
// NCPA::Units (src/common/units.cpp:120-260).  Produces SI knot arrays for
// ncpa_profile_create.
#pragma once

#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace ncpa {

struct ParsedProfile {
    std::vector<double> z;                      // altitude column as read
    std::string z_units;                        // canonical unit token
    std::map<std::string, std::vector<double>> vectors;
    std::map<std::string, std::string> vector_units;
    std::map<std::string, double> scalars;
    std::map<std::string, std::string> scalar_units;
};

struct ParseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// canonical unit token ("km", "m", "m/s", "K", "Pa", "mbar", "kg/m3", ...)
// for a units string of the profile header; throws ParseError if unknown
std::string canonical_units(const std::string& s);
// convert values in place to the SI unit named by target ("m", "m/s", "K",
// "Pa", "kg/m3"); throws ParseError if no conversion exists
void to_si(std::vector<double>& v, const std::string& from, const std::string& target);
double to_si(double v, const std::string& from, const std::string& target);

ParsedProfile read_profile(const std::string& path, const std::string& header_path);

// SI knot arrays ready for upload
struct SiProfile {
    std::vector<double> z, u, v, t, p, rho, c0, attn;
    bool has_c0 = false;
    double z0 = 0.0;
    bool has_z0 = false;
};
// the property checks and conversions of ESSModeSolver::setParams
// (ESSModeSolver.cpp:159-220); throws ParseError with the reference's message
SiProfile to_si_profile(const ParsedProfile& prof);

// G2S-style profile text (the layout of the reference's
// samples/g2sprofile.sample): an optional first line "Profile at (lat, lon)",
// '#' comment lines, then rows of at least six columns
//   Z [km]  T [K]  U [m/s]  V [m/s]  P [mbar]  RHO [g/cm3]
// (further columns ignored).  The reference's Atmosphere1D reads only
// "#%"-described files, so this is the conversion step in front of it.
// Returns the profile as if read from the equivalent NCPA file; lat / lon are
// NaN when the file has no location line.
ParsedProfile read_g2s_profile(const std::string& path, double& lat, double& lon);
// writes an NCPA profile file ("#% col, KEY, units" header + columns) holding
// the altitude column, the given vector keys in order and the scalars
void write_ncpa_profile(const ParsedProfile& prof, const std::vector<std::string>& keys, const std::string& path);

// two-column attenuation file (height km, Np/m), extended to the profile's
// range with end values (Atmosphere1D::read_attenuation_from_file,
// Atmosphere1D.cpp:307-424); returns (z_km, attn)
void read_attn_file(const std::string& path, std::vector<double>& z_km, std::vector<double>& a);

}  // namespace ncpa
