// NCPA profile file reader (see atmosphere.hpp).
#include "atmosphere.hpp"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <set>
#include <sstream>

namespace ncpa {

namespace {

std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

std::vector<std::string> split(const std::string& s, const char* delims) {
    std::vector<std::string> out;
    std::string cur;
    for (char ch : s) {
        if (std::strchr(delims, ch)) {
            if (!cur.empty()) out.push_back(cur);
            cur.clear();
        } else {
            cur.push_back(ch);
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

std::string upper(std::string s) {
    for (auto& c : s) c = (char)std::toupper((unsigned char)c);
    return s;
}

double parse_double(const std::string& tok, const std::string& line) {
    size_t pos = 0;
    double v;
    try {
        v = std::stod(tok, &pos);
    } catch (const std::exception&) {
        throw ParseError("Error parsing data line:\n" + line + "\nCan't parse field " + tok + " as a double");
    }
    if (pos != tok.size())
        throw ParseError("Error parsing data line:\n" + line + "\nCan't parse field " + tok + " as a double");
    return v;
}

}  // namespace

std::string canonical_units(const std::string& s) {
    static const std::map<std::string, std::string> table = {
        {"", ""}, {"N/A", ""},
        {"K", "K"}, {"DEGK", "K"}, {"DEG K", "K"}, {"DEGREES K", "K"}, {"KELVIN", "K"},
        {"C", "C"}, {"DEGC", "C"}, {"DEG C", "C"}, {"DEGREES C", "C"}, {"CELSIUS", "C"}, {"CENTIGRADE", "C"},
        {"F", "F"}, {"DEGF", "F"}, {"DEG F", "F"}, {"DEGREES F", "F"}, {"FAHRENHEIT", "F"},
        {"M", "m"}, {"METERS", "m"}, {"KM", "km"}, {"KILOMETERS", "km"},
        {"M/S", "m/s"}, {"MPS", "m/s"}, {"MPERS", "m/s"}, {"M PER S", "m/s"}, {"METERS PER SECOND", "m/s"},
        {"KM/S", "km/s"}, {"KMPS", "km/s"}, {"KMPERS", "km/s"}, {"KM PER S", "km/s"},
        {"KILOMETERS PER SECOND", "km/s"},
        {"PA", "Pa"}, {"PASCAL", "Pa"}, {"PASCALS", "Pa"},
        {"MBAR", "mbar"}, {"MILLIBAR", "mbar"}, {"MILLIBARS", "mbar"},
        {"HECTOPASCALS", "hPa"}, {"HPA", "hPa"}, {"ATMOSPHERES", "atm"}, {"ATM", "atm"},
        {"KG/M3", "kg/m3"}, {"KGPM3", "kg/m3"}, {"KILOGRAMS PER CUBIC METER", "kg/m3"},
        {"G/CM3", "g/cm3"}, {"GPCM3", "g/cm3"}, {"GRAMS PER CUBIC CENTIMETER", "g/cm3"},
        {"DEG", "deg"}, {"DEGREES", "deg"}, {"RAD", "rad"}, {"RADIANS", "rad"},
    };
    auto it = table.find(upper(s));
    if (it == table.end()) throw ParseError("Unrecognized units string: " + s);
    return it->second;
}

double to_si(double x, const std::string& from, const std::string& target) {
    if (from == target) return x;
    // same operations as the conversion table of units.cpp:132-172
    if (from == "km" && target == "m") return x * 1000.0;
    if (from == "m" && target == "km") return x * 0.001;
    if (from == "km/s" && target == "m/s") return x * 1000.0;
    if (from == "mbar" && target == "Pa") return x * 100.0;
    if (from == "hPa" && target == "Pa") return x * 100;
    if (from == "atm" && target == "Pa") return x * 101325.0;
    if (from == "g/cm3" && target == "kg/m3") return x * 1000.0;
    if (from == "C" && target == "K") return x + 273.15;
    if (from == "F" && target == "K") return ((x - 32.0) * 5.0 / 9.0) + 273.15;
    throw ParseError("No conversion from '" + from + "' to '" + target + "'");
}

void to_si(std::vector<double>& v, const std::string& from, const std::string& target) {
    for (auto& x : v) x = to_si(x, from, target);
}

ParsedProfile read_profile(const std::string& path, const std::string& header_path) {
    const std::string hfile = header_path.empty() ? path : header_path;
    std::vector<std::string> headerlines, datalines;
    {
        std::ifstream in(hfile);
        if (!in.good()) throw ParseError("Atmosphere1D - Input stream not in good state: " + hfile);
        std::string line;
        while (std::getline(in, line)) {
            line = trim(line);
            if (line.size() > 1 && line[0] == '#' && line[1] == '%') headerlines.push_back(line.substr(2));
        }
    }
    {
        std::ifstream in(path);
        if (!in.good()) throw ParseError("Atmosphere1D - Input stream not in good state: " + path);
        std::string line;
        while (std::getline(in, line)) {
            line = trim(line);
            if (line.empty() || line[0] == '#') continue;
            datalines.push_back(line);
        }
    }
    if (headerlines.empty()) throw ParseError("Atmosphere1D - No descriptive fields found.");
    std::vector<int> cols;
    std::vector<std::string> keys, units;
    std::vector<double> vals;
    for (const auto& h : headerlines) {
        auto f = split(trim(h), " ,");
        if (f.size() != 3 && f.size() != 4)
            throw ParseError("Atmosphere1D - Error parsing descriptive line:\n" + h +
                             "\nMust be formatted as:\ncolumn,key,units[,value]");
        int col;
        try {
            col = std::stoi(f[0]);
        } catch (const std::exception&) {
            throw ParseError("Atmosphere1D - Error parsing descriptive line:\n" + h +
                             "\nFirst field not parseable as an integer");
        }
        cols.push_back(col);
        keys.push_back(trim(f[1]));
        units.push_back(canonical_units(trim(f[2])));
        vals.push_back(f.size() == 4 ? parse_double(trim(f[3]), h) : 0.0);
    }
    {
        std::set<std::string> uk(keys.begin(), keys.end());
        if (uk.size() != keys.size()) throw ParseError("Atmosphere1D: key values are not unique");
    }
    int ncols = 0;
    std::string depunits;
    for (size_t i = 0; i < cols.size(); ++i) {
        ncols = std::max(ncols, cols[i]);
        if (cols[i] == 1) depunits = units[i];
    }
    std::vector<std::vector<double>> columns(ncols, std::vector<double>(datalines.size()));
    for (size_t r = 0; r < datalines.size(); ++r) {
        auto f = split(datalines[r], " \t,");
        if ((int)f.size() != ncols) {
            std::ostringstream os;
            os << "Error parsing data line:\n" << datalines[r] << "\n" << ncols << " columns expected, " << f.size()
               << " columns found.";
            throw ParseError(os.str());
        }
        for (int c = 0; c < ncols; ++c) columns[c][r] = parse_double(f[c], datalines[r]);
    }
    ParsedProfile P;
    if (ncols < 1) throw ParseError("Atmosphere1D - no altitude column");
    P.z = columns[0];
    P.z_units = depunits;
    for (size_t i = 0; i < keys.size(); ++i) {
        if (cols[i] == 0) {
            P.scalars[keys[i]] = vals[i];
            P.scalar_units[keys[i]] = units[i];
        } else if (cols[i] > 1) {
            P.vectors[keys[i]] = columns[cols[i] - 1];
            P.vector_units[keys[i]] = units[i];
        }
    }
    return P;
}

ParsedProfile read_g2s_profile(const std::string& path, double& lat, double& lon) {
    lat = lon = std::nan("");
    std::ifstream in(path);
    if (!in.good()) throw ParseError("G2S profile - cannot open " + path);
    static const char* const kKeys[] = {"T", "U", "V", "P", "RHO"};
    static const char* const kUnits[] = {"K", "m/s", "m/s", "mbar", "g/cm3"};
    ParsedProfile P;
    std::vector<std::vector<double>> cols(5);
    std::string line;
    bool first = true;
    while (std::getline(in, line)) {
        line = trim(line);
        if (line.empty() || line[0] == '#') continue;
        if (first && upper(line).rfind("PROFILE AT", 0) == 0) {
            const size_t a = line.find('('), b = line.find(')');
            if (a != std::string::npos && b != std::string::npos && b > a) {
                auto f = split(line.substr(a + 1, b - a - 1), " ,");
                if (f.size() == 2) {
                    lat = parse_double(f[0], line);
                    lon = parse_double(f[1], line);
                }
            }
            first = false;
            continue;
        }
        first = false;
        auto f = split(line, " \t,");
        if (f.size() < 6) {
            std::ostringstream os;
            os << "Error parsing data line:\n" << line << "\n6 columns expected (Z T U V P RHO), " << f.size()
               << " columns found.";
            throw ParseError(os.str());
        }
        P.z.push_back(parse_double(f[0], line));
        for (int c = 0; c < 5; ++c) cols[c].push_back(parse_double(f[c + 1], line));
    }
    if (P.z.size() < 3) throw ParseError("G2S profile - fewer than 3 data rows in " + path);
    P.z_units = canonical_units("km");
    for (int c = 0; c < 5; ++c) {
        P.vectors[kKeys[c]] = cols[c];
        P.vector_units[kKeys[c]] = canonical_units(kUnits[c]);
    }
    return P;
}

void write_ncpa_profile(const ParsedProfile& prof, const std::vector<std::string>& keys, const std::string& path) {
    std::ofstream out(path);
    if (!out.good()) throw ParseError("cannot write " + path);
    int col = 0;
    for (const auto& kv : prof.scalars) {
        auto u = prof.scalar_units.find(kv.first);
        char buf[256];
        std::snprintf(buf, sizeof buf, "#%% 0, %s, %s, %.17g\n", kv.first.c_str(),
                      u == prof.scalar_units.end() || u->second.empty() ? "N/A" : u->second.c_str(), kv.second);
        out << buf;
    }
    out << "#% " << ++col << ", Z, " << prof.z_units << "\n";
    for (const auto& k : keys) {
        auto u = prof.vector_units.find(k);
        if (prof.vectors.find(k) == prof.vectors.end()) throw ParseError("no column " + k + " to write");
        out << "#% " << ++col << ", " << k << ", " << (u == prof.vector_units.end() ? "N/A" : u->second) << "\n";
    }
    char buf[64];
    for (size_t r = 0; r < prof.z.size(); ++r) {
        std::snprintf(buf, sizeof buf, "%.17g", prof.z[r]);
        out << buf;
        for (const auto& k : keys) {
            std::snprintf(buf, sizeof buf, " %.17g", prof.vectors.at(k)[r]);
            out << buf;
        }
        out << "\n";
    }
    if (!out.good()) throw ParseError("error writing " + path);
}

SiProfile to_si_profile(const ParsedProfile& prof) {
    SiProfile S;
    if (prof.z.size() < 3) throw ParseError("Atmosphere1D - need at least 3 altitude points");
    S.z = prof.z;
    to_si(S.z, prof.z_units, "m");
    for (size_t i = 1; i < S.z.size(); ++i)
        if (!(S.z[i] > S.z[i - 1])) throw ParseError("Atmosphere1D - altitudes must increase strictly");
    auto get = [&](const char* key, const char* target, std::vector<double>& out) -> bool {
        auto it = prof.vectors.find(key);
        if (it == prof.vectors.end()) return false;
        out = it->second;
        to_si(out, prof.vector_units.at(key), target);
        return true;
    };
    if (get("C0", "m/s", S.c0)) S.has_c0 = true;
    const bool hasP = prof.vectors.count("P") > 0, hasR = prof.vectors.count("RHO") > 0,
               hasT = prof.vectors.count("T") > 0;
    if (!S.has_c0 && !(hasP && hasR) && !hasT)
        throw ParseError(
            "Can't calculate static sound speed, either temperature T or pressure P and density RHO missing");
    if (!get("U", "m/s", S.u)) throw ParseError("U wind vector not found in atmosphere file");
    if (!get("V", "m/s", S.v)) throw ParseError("V wind vector not found in atmosphere file");
    if (!get("T", "K", S.t)) {
        if (!S.has_c0) throw ParseError("T temperature vector not found in atmosphere file");
        // temperature from the user sound speed (Atmosphere1D.cpp:794-818)
        S.t.resize(S.c0.size());
        for (size_t i = 0; i < S.c0.size(); ++i) S.t[i] = S.c0[i] * S.c0[i] / 1.4 / 287.0;
    }
    if (!get("P", "Pa", S.p)) throw ParseError("P pressure vector not found in atmosphere file");
    if (!get("RHO", "kg/m3", S.rho)) throw ParseError("RHO density vector not found in atmosphere file");
    auto z0 = prof.scalars.find("Z0");
    if (z0 != prof.scalars.end()) {
        S.z0 = to_si(z0->second, prof.scalar_units.at("Z0"), "m");
        S.has_z0 = true;
    }
    return S;
}

void read_attn_file(const std::string& path, std::vector<double>& z_km, std::vector<double>& a) {
    std::ifstream in(path);
    if (!in.good()) throw ParseError("attenuation file " + path + " could not be opened");
    std::string line;
    z_km.clear();
    a.clear();
    while (std::getline(in, line)) {
        line = trim(line);
        if (line.empty() || line[0] == '#') continue;
        auto f = split(line, " ,");
        if (f.size() != 2)
            throw ParseError("Atmosphere1D - Error parsing attenuation line:\n" + line +
                             "\nMust be formatted as:\naltitude  attenuation");
        z_km.push_back(parse_double(f[0], line));
        a.push_back(parse_double(f[1], line));
    }
    if (z_km.size() < 2) throw ParseError("attenuation file " + path + " needs at least two rows");
}

}  // namespace ncpa
