// Boost-free configuration parser with the reference's semantics
// (include/bohrium/bh_config_parser.hpp:86-298, core/bh_config_parser.cpp:44-232):
//  - the config file is found via $BH_CONFIG, then ~/.bohrium/config.ini, then the system paths;
//  - the stack is the comma/space separated list `[stacks] <BH_STACK or "default">`;
//  - every option can be overridden by the environment variable BH_<SECTION>_<OPTION>
//    (upper case, '-' and ' ' replaced by '_');
//  - values may be quoted; "{CONF_PATH}" expands to the config file's directory;
//  - booleans accept y/n/t/f/1/0 by their first character.
#pragma once

#include <cstdint>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <typeinfo>
#include <vector>

namespace bohrium {

class ConfigError : public std::exception {
    std::string _msg;

public:
    explicit ConfigError(std::string msg) : _msg(std::move(msg)) {}
    const char *what() const noexcept override { return _msg.c_str(); }
};
class ConfigNoChild : public ConfigError {
public:
    explicit ConfigNoChild(const std::string &msg) : ConfigError(msg) {}
};
class ConfigKeyNotFound : public ConfigError {
public:
    explicit ConfigKeyNotFound(const std::string &msg) : ConfigError(msg) {}
};
class ConfigBadCast : public ConfigError {
public:
    explicit ConfigBadCast(const std::string &msg) : ConfigError(msg) {}
};

namespace config_detail {
template <typename T>
inline T lexical(const std::string &s) {
    std::stringstream ss(s);
    T v;
    ss >> v;
    if (ss.fail() || !(ss >> std::ws).eof()) throw std::invalid_argument(s);
    return v;
}
template <>
inline std::string lexical<std::string>(const std::string &s) { return s; }
template <>
inline bool lexical<bool>(const std::string &s) {
    if (s.empty()) throw std::invalid_argument(s);
    switch (s[0]) {
        case 'y': case 'Y': case '1': case 't': case 'T': return true;
        case 'n': case 'N': case '0': case 'f': case 'F': return false;
        default: throw std::invalid_argument(s);
    }
}
} // namespace config_detail

class ConfigParser {
public:
    const std::string file_path;
    const std::string file_dir; // directory of the config file, with a trailing '/'
    const int stack_level;

private:
    std::string _default_section;
    std::vector<std::string> _stack_list;
    std::map<std::string, std::map<std::string, std::string>> _config; // section -> option -> value
    std::string lookup(const std::string &section, const std::string &option) const;

public:
    // Locate the config file and the stack like the reference does.
    explicit ConfigParser(int stack_level);
    // Use an explicit config file and stack name (empty strings fall back to the search above).
    ConfigParser(int stack_level, const std::string &config_path, const std::string &stack_name);

    std::string expand(const std::string &path) const;

    template <typename T>
    T get(const std::string &section, const std::string &option) const {
        std::string ret = lookup(section, option);
        const std::string key = "{CONF_PATH}";
        for (size_t p = ret.find(key); p != std::string::npos; p = ret.find(key)) ret.replace(p, key.size(), file_dir);
        try {
            return config_detail::lexical<T>(ret);
        } catch (const std::exception &) {
            throw ConfigBadCast("ConfigParser cannot convert '" + section + "." + option + "=" + ret + "' to type <" +
                                typeid(T).name() + ">");
        }
    }
    template <typename T>
    T get(const std::string &option) const { return get<T>(_default_section, option); }
    template <typename T>
    T defaultGet(const std::string &section, const std::string &option, const T &default_value) const {
        try {
            return get<T>(section, option);
        } catch (const ConfigKeyNotFound &) {
            return default_value;
        }
    }
    template <typename T>
    T defaultGet(const std::string &option, const T &default_value) const {
        return defaultGet<T>(_default_section, option, default_value);
    }
    std::vector<std::string> getList(const std::string &section, const std::string &option) const;
    std::vector<std::string> getList(const std::string &option) const { return getList(_default_section, option); }
    std::vector<std::string> defaultGetList(const std::string &option, const std::vector<std::string> &def) const;
    // Like getList() but each entry is a path; relative paths are taken relative to the config file.
    std::vector<std::string> getListOfPaths(const std::string &section, const std::string &option) const;
    std::vector<std::string> getListOfPaths(const std::string &option) const {
        return getListOfPaths(_default_section, option);
    }
    // A path option resolved like getListOfPaths() does for each entry.
    std::string getPath(const std::string &section, const std::string &option) const;
    // Library path of the next component in the stack, or "" when this is the last one.
    std::string getChildLibraryPath() const;
    const std::string &getName() const { return _default_section; }
    const std::vector<std::string> &getStackList() const { return _stack_list; }
};

} // namespace bohrium
