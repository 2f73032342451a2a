/*
 * Minimal stand-in for <boost/program_options.hpp>, used ONLY to compile the
 * reference solver's Options class into the CPU oracle binary (oracle/_ref).
 * Test infrastructure: never linked into the product library.
 *
 * Covers the subset the reference uses: options_description + add_options()
 * with po::value<T>(&target), parse_config_file on an INI stream
 * ("[SECTION]" headers prefix keys as "SECTION.KEY", '#' comments,
 * "key = value" lines), store, notify and variables_map::count.
 * Unknown keys raise, as boost does without allow_unregistered.
 */
#ifndef MC3D_ORACLE_BOOST_PO_SHIM_HPP
#define MC3D_ORACLE_BOOST_PO_SHIM_HPP

#include <algorithm>
#include <istream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace boost {
namespace program_options {

struct value_semantic {
    virtual ~value_semantic() {}
    virtual void assign(const std::string &text) = 0;
};

template <typename T>
struct typed_value : value_semantic {
    T *target;
    explicit typed_value(T *t) : target(t) {}
    void assign(const std::string &text) override {
        std::istringstream is(text);
        T v;
        is >> v;
        if (is.fail()) throw std::runtime_error("invalid option value: " + text);
        *target = v;
    }
};

template <>
struct typed_value<std::string> : value_semantic {
    std::string *target;
    explicit typed_value(std::string *t) : target(t) {}
    void assign(const std::string &text) override { *target = text; }
};

template <>
struct typed_value<bool> : value_semantic {
    bool *target;
    explicit typed_value(bool *t) : target(t) {}
    void assign(const std::string &text) override {
        std::string s = text;
        std::transform(s.begin(), s.end(), s.begin(), ::tolower);
        if (s == "1" || s == "true" || s == "yes" || s == "on") *target = true;
        else if (s == "0" || s == "false" || s == "no" || s == "off") *target = false;
        else throw std::runtime_error("invalid bool option value: " + text);
    }
};

template <typename T>
typed_value<T> *value(T *target) { return new typed_value<T>(target); }

class options_description;

struct options_init {
    options_description *owner;
    options_init &operator()(const char *name, value_semantic *v, const char *desc = "");
};

class options_description {
  public:
    explicit options_description(const std::string & = "") {}
    options_init add_options() { return options_init{this}; }
    std::map<std::string, std::shared_ptr<value_semantic> > opts;
};

inline options_init &options_init::operator()(const char *name, value_semantic *v, const char *) {
    owner->opts[name] = std::shared_ptr<value_semantic>(v);
    return *this;
}

struct parsed_options {
    const options_description *desc;
    std::vector<std::pair<std::string, std::string> > items;
};

inline std::string mc3d_trim(const std::string &s) {
    size_t a = s.find_first_not_of(" \t\r\n");
    if (a == std::string::npos) return "";
    size_t b = s.find_last_not_of(" \t\r\n");
    return s.substr(a, b - a + 1);
}

inline parsed_options parse_config_file(std::istream &is, const options_description &desc,
                                        bool allow_unregistered = false) {
    parsed_options p;
    p.desc = &desc;
    std::string line, prefix;
    while (std::getline(is, line)) {
        size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        line = mc3d_trim(line);
        if (line.empty()) continue;
        if (line[0] == '[') {
            size_t e = line.find(']');
            prefix = mc3d_trim(line.substr(1, e - 1)) + ".";
            continue;
        }
        size_t eq = line.find('=');
        if (eq == std::string::npos) throw std::runtime_error("syntax error: " + line);
        std::string key = prefix + mc3d_trim(line.substr(0, eq));
        std::string val = mc3d_trim(line.substr(eq + 1));
        if (!desc.opts.count(key)) {
            if (allow_unregistered) continue;
            throw std::runtime_error("unrecognised option '" + key + "'");
        }
        p.items.push_back(std::make_pair(key, val));
    }
    return p;
}

class variables_map {
  public:
    size_t count(const std::string &k) const { return vals.count(k); }
    std::map<std::string, std::string> vals;
    const options_description *desc = nullptr;
};

inline void store(const parsed_options &p, variables_map &vm) {
    vm.desc = p.desc;
    for (auto &kv : p.items)
        if (!vm.vals.count(kv.first)) vm.vals[kv.first] = kv.second;
}

inline void notify(variables_map &vm) {
    if (!vm.desc) return;
    for (auto &kv : vm.vals) vm.desc->opts.at(kv.first)->assign(kv.second);
}

}  // namespace program_options
}  // namespace boost

#endif
