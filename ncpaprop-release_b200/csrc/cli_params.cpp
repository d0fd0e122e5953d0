// Option parsing of the front ends (see cli_params.hpp).
#include "cli_params.hpp"

#include <cctype>
#include <cstring>
#include <fstream>
#include <sstream>

namespace ncpa_cli {

namespace {
std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}
bool is_long(const std::string& o) { return o.size() >= 3 && o.compare(0, 2, "--") == 0; }
bool is_short(const std::string& o) {
    return o.size() >= 2 && o[0] == '-' && o[1] != '-' && !std::isdigit((unsigned char)o[1]);
}
std::string num(double v) { return std::to_string(v); }
enum { T_REQ, T_REQIF, T_FGT, T_FGE, T_FLT, T_FLE, T_IGT, T_IGE, T_SET, T_RADIO };
}  // namespace

Params::P& Params::at(const std::string& key) {
    auto it = params_.find(key);
    if (it == params_.end()) throw OptionError("Unknown parameter '" + key + "'");
    return it->second;
}
const Params::P& Params::at(const std::string& key) const {
    auto it = params_.find(key);
    if (it == params_.end()) throw OptionError("Unknown parameter '" + key + "'");
    return it->second;
}

void Params::add_flag(const std::string& key, bool dflt) {
    P p;
    p.kind = FLAG;
    p.found = dflt;
    p.valid = true;
    params_[key] = p;
    order_.push_back(key);
}
void Params::add_string(const std::string& key, const std::string& dflt, bool has_default) {
    P p;
    p.kind = STRING;
    p.sval = dflt;
    p.valid = has_default;
    params_[key] = p;
    order_.push_back(key);
}
void Params::add_float(const std::string& key, double dflt, bool has_default) {
    P p;
    p.kind = FLOAT;
    p.fval = dflt;
    p.valid = has_default;
    params_[key] = p;
    order_.push_back(key);
}
void Params::add_int(const std::string& key, int dflt) {
    P p;
    p.kind = INT;
    p.ival = dflt;
    p.valid = true;
    params_[key] = p;
    order_.push_back(key);
}

void Params::require(const std::string& key) { tests_.push_back({T_REQ, key, "", 0.0, {}}); }
void Params::require_if(const std::string& key, const std::string& other) {
    tests_.push_back({T_REQIF, key, other, 0.0, {}});
}
void Params::float_gt(const std::string& key, double v) { tests_.push_back({T_FGT, key, "", v, {}}); }
void Params::float_ge(const std::string& key, double v) { tests_.push_back({T_FGE, key, "", v, {}}); }
void Params::float_lt(const std::string& key, double v) { tests_.push_back({T_FLT, key, "", v, {}}); }
void Params::float_le(const std::string& key, double v) { tests_.push_back({T_FLE, key, "", v, {}}); }
void Params::int_gt(const std::string& key, int v) { tests_.push_back({T_IGT, key, "", (double)v, {}}); }
void Params::int_ge(const std::string& key, int v) { tests_.push_back({T_IGE, key, "", (double)v, {}}); }
void Params::string_set(const std::string& key, const std::vector<std::string>& choices) {
    tests_.push_back({T_SET, key, "", 0.0, choices});
}
void Params::radio(const std::string& name, const std::vector<std::string>& buttons) {
    tests_.push_back({T_RADIO, name, "", 0.0, buttons});
}

void Params::single(const std::string& key) {
    auto it = params_.find(key);
    if (it == params_.end()) throw OptionError("Unexpected argument: '" + key + "'");
    if (it->second.kind != FLAG)
        throw OptionError("Option " + key + " expects an argument, but none appears to be provided.");
    it->second.found = true;
}

void Params::dbl(const std::string& key, const std::string& value) {
    auto it = params_.find(key);
    if (it == params_.end()) throw OptionError("Unexpected argument: '" + key + "'");
    P& p = it->second;
    if (p.kind == FLAG)
        throw OptionError("Option " + key + " appears to have an argument '" + value + "', but is not expecting one.");
    try {
        size_t pos = 0;
        if (p.kind == FLOAT) {
            p.fval = std::stod(value, &pos);
        } else if (p.kind == INT) {
            p.ival = std::stoi(value, &pos);
        } else {
            p.sval = value;
            pos = value.size();
        }
        if (pos != value.size()) throw std::invalid_argument("trailing characters");
    } catch (const std::exception&) {
        throw OptionError("Can't parse '" + value + "' as a value of option " + key);
    }
    p.found = true;
    p.valid = true;
}

void Params::parse_command_line(int argc, char** argv) {
    for (int i = 1; i < argc; ++i) {
        std::string arg = argv[i];
        if (is_long(arg)) {
            std::string stripped = arg.substr(arg.find_first_not_of('-'));
            size_t d = stripped.find_first_of(delims_);
            if (d != std::string::npos) {
                dbl(stripped.substr(0, d), stripped.substr(d + 1));
                continue;
            }
            auto it = params_.find(stripped);
            if (it == params_.end()) throw OptionError("Unknown option '" + arg + "'.");
            if (it->second.kind == FLAG) {
                single(stripped);
            } else {
                if (i + 1 >= argc)
                    throw OptionError("Option '" + stripped + "' expects a value, but none was provided.");
                std::string value = argv[i + 1];
                if (is_long(value) || is_short(value))
                    throw OptionError("Value '" + value + "' for option '" + stripped +
                                      "' appears to be another argument.");
                dbl(stripped, value);
                ++i;
            }
        } else if (is_short(arg)) {
            std::string stripped = arg.substr(arg.find_first_not_of('-'));
            for (char ch : stripped) {
                std::string k(1, ch);
                if (!params_.count(k)) throw OptionError("Unexpected argument '-" + k + "'.");
                params_[k].found = true;
            }
        }
        // other words are ignored, as the reference keeps them as unparsed
    }
}

void Params::parse_file(const std::string& path) {
    std::ifstream in(path);
    if (!in.good()) return;
    std::string line;
    while (std::getline(in, line)) {
        line = trim(line);
        if (line.empty() || line[0] == '#' || line[0] == '%') continue;
        std::vector<std::string> tok;
        std::string cur;
        for (char ch : line) {
            if (std::strchr(delims_, ch)) {
                if (!cur.empty()) tok.push_back(cur);
                cur.clear();
            } else {
                cur.push_back(ch);
            }
        }
        if (!cur.empty()) tok.push_back(cur);
        if (tok.size() > 2) throw OptionError("Ambiguous line in file " + path + ": '" + line + "'.");
        if (tok.size() == 1) single(trim(tok[0]));
        else if (tok.size() == 2) dbl(trim(tok[0]), trim(tok[1]));
    }
}

bool Params::validate(std::ostream& os) const {
    bool ok = true;
    for (const Test& t : tests_) {
        bool pass = true;
        std::string msg;
        if (t.type == T_RADIO) {
            int n = 0;
            std::string vs = "{ ";
            for (size_t i = 0; i < t.set.size(); ++i) {
                if (found(t.set[i])) ++n;
                vs += t.set[i] + (i + 1 < t.set.size() ? ", " : " }");
            }
            pass = n == 1;
            msg = t.key + ": " + std::to_string(n) + " of " + vs + " are present; must be one and only one.";
        } else if (t.type == T_REQ) {
            pass = found(t.key);
            msg = t.key + " is not present.";
        } else if (t.type == T_REQIF) {
            pass = !found(t.other) || found(t.key);
            msg = "One of { " + t.other + " } is set, but " + t.key + " is not set.";
        } else {
            const P& p = at(t.key);
            if (!p.valid) continue;
            if (t.type == T_SET) {
                pass = false;
                std::string vs = "{ ";
                for (size_t i = 0; i < t.set.size(); ++i) {
                    if (p.sval == t.set[i]) pass = true;
                    vs += t.set[i] + (i + 1 < t.set.size() ? ", " : " }");
                }
                msg = t.key + ": \"" + p.sval + "\" is not in " + vs + ".";
            } else if (t.type == T_IGT || t.type == T_IGE) {
                const double x = p.kind == INT ? p.ival : p.fval;
                pass = t.type == T_IGT ? x > t.v : x >= t.v;
                msg = t.key + " (" + std::to_string((long long)x) + ") must be greater than " +
                      (t.type == T_IGE ? std::string("or equal to ") : std::string()) +
                      std::to_string((long long)t.v) + ".";
            } else {
                const double x = p.kind == INT ? p.ival : p.fval;
                switch (t.type) {
                    case T_FGT: pass = x > t.v; msg = t.key + " (" + num(x) + ") must be greater than " + num(t.v) + "."; break;
                    case T_FGE: pass = x >= t.v; msg = t.key + " (" + num(x) + ") must be greater than or equal to " + num(t.v) + "."; break;
                    case T_FLT: pass = x < t.v; msg = t.key + " (" + num(x) + ") must be less than " + num(t.v) + "."; break;
                    default: pass = x <= t.v; msg = t.key + " (" + num(x) + ") must be less than " + num(t.v) + "."; break;
                }
            }
        }
        if (!pass) {
            os << msg << "\n";
            ok = false;
        }
    }
    return ok;
}

bool Params::found(const std::string& key) const {
    auto it = params_.find(key);
    return it != params_.end() && it->second.found;
}
bool Params::get_bool(const std::string& key) const {
    const P& p = at(key);
    if (p.kind == FLAG) return p.found;
    return p.valid;
}
double Params::get_float(const std::string& key) const {
    const P& p = at(key);
    if (!p.valid) throw OptionError("Parameter " + key + " not set");
    return p.kind == INT ? p.ival : p.fval;
}
int Params::get_int(const std::string& key) const {
    const P& p = at(key);
    if (!p.valid) throw OptionError("Parameter " + key + " not set");
    return p.kind == FLOAT ? (int)p.fval : p.ival;
}
std::string Params::get_string(const std::string& key) const {
    const P& p = at(key);
    if (!p.valid) return "";
    if (p.kind == FLAG) return p.found ? "true" : "false";
    return p.sval;
}

void Params::print(std::ostream& os) const {
    for (const auto& k : order_) {
        const P& p = params_.at(k);
        os << k << ": ";
        if (p.kind == FLAG) os << (p.found ? "true" : "false");
        else if (!p.valid) os << "(not set)";
        else if (p.kind == FLOAT) os << p.fval;
        else if (p.kind == INT) os << p.ival;
        else os << p.sval;
        os << "\n";
    }
}

}  // namespace ncpa_cli
