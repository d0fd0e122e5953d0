// Command-line / parameter-file options of the Modess and ModBB front ends:
// the syntax and validation of NCPA::ParameterSet (src/common/parameterset.cpp
// :322-594): "--key value", "--key=value" (any of the delimiters "=: "),
// "--flag", short flags "-h", a parameter file of "key: value" lines read
// between two command-line passes, strict mode, and the tests the front ends
// register (required, required-if-other-present, numeric bounds, string
// sets, radio buttons).
#pragma once

#include <map>
#include <ostream>
#include <stdexcept>
#include <string>
#include <vector>

namespace ncpa_cli {

struct OptionError : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};

class Params {
public:
    enum Kind { FLAG, STRING, FLOAT, INT };

    void add_flag(const std::string& key, bool dflt = false);
    void add_string(const std::string& key, const std::string& dflt, bool has_default = true);
    void add_string_nodefault(const std::string& key) { add_string(key, "", false); }
    void add_float(const std::string& key, double dflt, bool has_default = true);
    void add_float_nodefault(const std::string& key) { add_float(key, 0.0, false); }
    void add_int(const std::string& key, int dflt);

    // tests
    void require(const std::string& key);
    void require_if(const std::string& key, const std::string& other);
    void float_gt(const std::string& key, double v);
    void float_ge(const std::string& key, double v);
    void float_lt(const std::string& key, double v);
    void float_le(const std::string& key, double v);
    void int_gt(const std::string& key, int v);
    void int_ge(const std::string& key, int v);
    void string_set(const std::string& key, const std::vector<std::string>& choices);
    void radio(const std::string& name, const std::vector<std::string>& buttons);

    void parse_command_line(int argc, char** argv);  // throws OptionError
    void parse_file(const std::string& path);        // missing file: ignored
    bool validate(std::ostream& failures) const;

    bool found(const std::string& key) const;
    bool get_bool(const std::string& key) const;
    double get_float(const std::string& key) const;
    int get_int(const std::string& key) const;
    std::string get_string(const std::string& key) const;
    void print(std::ostream& os) const;

private:
    struct P {
        Kind kind = FLAG;
        bool found = false;
        bool valid = false;  // has a value (default or given)
        std::string sval;
        double fval = 0.0;
        int ival = 0;
    };
    struct Test {
        int type;
        std::string key, other;
        double v = 0.0;
        std::vector<std::string> set;
    };
    std::map<std::string, P> params_;
    std::vector<std::string> order_;
    std::vector<Test> tests_;
    const char* delims_ = "=: ";

    P& at(const std::string& key);
    const P& at(const std::string& key) const;
    void single(const std::string& key);
    void dbl(const std::string& key, const std::string& value);
};

}  // namespace ncpa_cli
