// Command-line parsing for the index / search tools: the option spellings of
// the reference's tools (boost::program_options in index.cpp:42-83 and
// search.cpp:37-62): "--name value", "--name=value", "-K value", "-K10",
// flags without a value, and positional arguments in order.
#pragma once
#include <cctype>
#include <cstdlib>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

namespace kgcli {

struct Args {
    std::map<std::string, std::string> values;   // option name (long, or the short letter) -> value
    std::set<std::string> flags;
    std::vector<std::string> positional;

    bool has(const std::string &k) const { return values.count(k) || flags.count(k); }
    std::string str(const std::string &k, const std::string &def = "") const {
        auto it = values.find(k);
        return it == values.end() ? def : it->second;
    }
    unsigned u(const std::string &k, unsigned def) const {
        auto it = values.find(k);
        return it == values.end() ? def : (unsigned)std::strtoul(it->second.c_str(), nullptr, 10);
    }
    int i(const std::string &k, int def) const {
        auto it = values.find(k);
        return it == values.end() ? def : (int)std::strtol(it->second.c_str(), nullptr, 10);
    }
    float f(const std::string &k, float def) const {
        auto it = values.find(k);
        return it == values.end() ? def : std::strtof(it->second.c_str(), nullptr);
    }
};

// `with_value`: option names that take a value; `alias`: short letter -> long
// name (both spellings end up under the long name).  Anything else starting
// with '-' is a flag; an unknown option with a value is an error, as in the
// reference's parser.
inline Args parse(int argc, char **argv, const std::set<std::string> &with_value,
                  const std::map<std::string, std::string> &alias, const std::set<std::string> &flag_names) {
    Args a;
    auto canon = [&](std::string k) {
        auto it = alias.find(k);
        return it == alias.end() ? k : it->second;
    };
    for (int n = 1; n < argc; ++n) {
        std::string s = argv[n];
        if (s.size() > 1 && s[0] == '-' && !(s.size() > 1 && (std::isdigit((unsigned char)s[1]) || s[1] == '.'))) {
            std::string key, val;
            bool has_val = false;
            if (s.rfind("--", 0) == 0) {
                key = s.substr(2);
                size_t eq = key.find('=');
                if (eq != std::string::npos) { val = key.substr(eq + 1); key = key.substr(0, eq); has_val = true; }
            } else {
                key = s.substr(1, 1);
                if (s.size() > 2) { val = s.substr(2); has_val = true; }
            }
            key = canon(key);
            if (with_value.count(key)) {
                if (!has_val) {
                    if (n + 1 >= argc) throw std::invalid_argument("option --" + key + " needs a value");
                    val = argv[++n];
                }
                a.values[key] = val;
            } else if (flag_names.count(key)) {
                a.flags.insert(key);
            } else {
                throw std::invalid_argument("unrecognised option '" + s + "'");
            }
        } else {
            a.positional.push_back(s);
        }
    }
    return a;
}

}  // namespace kgcli
