// Config file parsing, the component loader and the extmethod loader.
// Behaviour follows core/bh_config_parser.cpp:44-232, core/bh_component.cpp:30-143 and
// core/bh_extmethod.cpp:33-101 of the reference (without Boost).
#include <algorithm>
#include <cctype>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <dlfcn.h>
#include <bohrium/bh_config_parser.hpp>
#include <bohrium/bh_component.hpp>
#include <bohrium/bh_extmethod.hpp>

using namespace std;

namespace bohrium {
namespace {

bool file_exists(const string &p) {
    FILE *fp = fopen(p.c_str(), "r");
    if (fp) fclose(fp);
    return fp != nullptr;
}

// $BH_CONFIG, then ~/.bohrium/config.ini, then the three system-wide locations.
string find_config_path() {
    const char *env = getenv("BH_CONFIG");
    if (env != nullptr && file_exists(env)) return env;
    const char *home = getenv("HOME");
    if (home != nullptr) {
        const string p = string(home) + "/.bohrium/config.ini";
        if (file_exists(p)) return p;
    }
    for (const char *p : {"/usr/local/etc/bohrium/config.ini", "/usr/etc/bohrium/config.ini", "/etc/bohrium/config.ini"})
        if (file_exists(p)) return p;
    throw invalid_argument(
        "Bohrium could not find the config file (searched $BH_CONFIG, ~/.bohrium/config.ini, "
        "/usr/local/etc/bohrium/config.ini, /usr/etc/bohrium/config.ini, /etc/bohrium/config.ini)");
}

string trim(const string &s) {
    size_t b = 0, e = s.size();
    while (b < e && isspace(static_cast<unsigned char>(s[b]))) ++b;
    while (e > b && isspace(static_cast<unsigned char>(s[e - 1]))) --e;
    return s.substr(b, e - b);
}

string dir_of(const string &path) {
    const size_t p = path.find_last_of('/');
    return p == string::npos ? string("./") : path.substr(0, p + 1);
}

// INI parsing: [section] headers, key = value lines, '#' and ';' comment lines.
map<string, map<string, string>> read_ini(const string &path) {
    ifstream in(path);
    if (!in) throw ConfigError("ConfigParser: cannot read '" + path + "'");
    map<string, map<string, string>> ret;
    string line, section;
    int lineno = 0;
    while (getline(in, line)) {
        ++lineno;
        const string t = trim(line);
        if (t.empty() || t[0] == '#' || t[0] == ';') continue;
        if (t[0] == '[') {
            const size_t e = t.find(']');
            if (e == string::npos) throw ConfigError("ConfigParser: bad section header at " + path + ":" + to_string(lineno));
            section = trim(t.substr(1, e - 1));
            ret[section];
            continue;
        }
        const size_t eq = t.find('=');
        if (eq == string::npos) throw ConfigError("ConfigParser: expected 'key = value' at " + path + ":" + to_string(lineno));
        ret[section][trim(t.substr(0, eq))] = trim(t.substr(eq + 1));
    }
    return ret;
}

string env_name(const string &section, const string &option) {
    string s = "BH_" + section + "_" + option;
    for (char &c : s) {
        c = static_cast<char>(toupper(static_cast<unsigned char>(c)));
        if (c == '-' || c == ' ') c = '_';
    }
    return s;
}

vector<string> split_list(const string &s) {
    vector<string> ret;
    string cur;
    for (char c : s) {
        if (c == ',' || c == ' ' || c == '\t') {
            if (!cur.empty()) ret.push_back(cur);
            cur.clear();
        } else {
            cur += c;
        }
    }
    if (!cur.empty()) ret.push_back(cur);
    return ret;
}

} // namespace

ConfigParser::ConfigParser(int stack_level) : ConfigParser(stack_level, "", "") {}

ConfigParser::ConfigParser(int level, const string &config_path, const string &stack_name)
    : file_path(config_path.empty() ? find_config_path() : config_path), file_dir(dir_of(file_path)),
      stack_level(level) {
    _config = read_ini(file_path);
    string name = stack_name;
    if (name.empty()) {
        const char *env = getenv("BH_STACK");
        name = env == nullptr ? "default" : env;
    }
    _stack_list = getList("stacks", name);
    if (stack_level >= static_cast<int>(_stack_list.size()) || stack_level < -1)
        throw ConfigError("ConfigParser: stack level is out of bound");
    _default_section = stack_level == -1 ? string("bridge") : _stack_list[stack_level];
}

string ConfigParser::lookup(const string &section, const string &option) const {
    const char *env = getenv(env_name(section, option).c_str());
    if (env != nullptr && env[0] != '\0') return env;
    auto s = _config.find(section);
    if (s == _config.end() || s->second.find(option) == s->second.end()) {
        throw ConfigKeyNotFound("Error parsing the config file '" + file_path + "': '" + section + "." + option +
                                "' not found!");
    }
    string ret = s->second.at(option);
    if (ret.size() >= 2 && (ret.front() == '"' || ret.front() == '\'') && (ret.back() == '"' || ret.back() == '\''))
        return ret.substr(1, ret.size() - 2);
    return ret;
}

string ConfigParser::expand(const string &path) const {
    if (path.empty() || path[0] != '~') return path;
    const char *home = getenv("HOME");
    if (home == nullptr) throw invalid_argument("Couldn't expand `~` since $HOME environment variable not set.");
    return string(home) + path.substr(1);
}

vector<string> ConfigParser::getList(const string &section, const string &option) const {
    return split_list(get<string>(section, option));
}

vector<string> ConfigParser::defaultGetList(const string &option, const vector<string> &def) const {
    try {
        return getList(option);
    } catch (const ConfigKeyNotFound &) {
        return def;
    }
}

vector<string> ConfigParser::getListOfPaths(const string &section, const string &option) const {
    vector<string> ret;
    for (const string &p : getList(section, option)) {
        const string e = expand(p);
        ret.push_back(e.empty() || e[0] == '/' ? e : file_dir + e);
    }
    return ret;
}

string ConfigParser::getPath(const string &section, const string &option) const {
    const string e = expand(get<string>(section, option));
    return e.empty() || e[0] == '/' ? e : file_dir + e;
}

string ConfigParser::getChildLibraryPath() const {
    if (static_cast<int>(_stack_list.size()) <= stack_level + 1) return string();
    return getPath(_stack_list[stack_level + 1], "impl");
}

// ---------------------------------------------------------------------------------------------
namespace component {

ComponentFace::ComponentFace(const string &lib_path, int stack_level) {
    _lib_handle = dlopen(lib_path.c_str(), RTLD_NOW);
    if (_lib_handle == nullptr) {
        throw runtime_error(string("ComponentFace: cannot load library: ") + dlerror());
    }
    dlerror();
    *reinterpret_cast<void **>(&_create) = dlsym(_lib_handle, "create");
    if (const char *err = dlerror()) throw runtime_error(string("ComponentFace: cannot load function 'create': ") + err);
    *reinterpret_cast<void **>(&_destroy) = dlsym(_lib_handle, "destroy");
    if (const char *err = dlerror()) throw runtime_error(string("ComponentFace: cannot load function 'destroy': ") + err);
    _implementation = _create(stack_level);
}

ComponentFace::~ComponentFace() {
    if (initiated()) {
        _destroy(_implementation);
        // Libraries stay mapped: CUDA and OpenMP runtimes register exit handlers inside them.
    }
}

bool ComponentFace::initiated() const { return _implementation != nullptr; }

#define BH_REQUIRE_INIT() \
    if (!initiated()) throw std::runtime_error("uninitiated component interface")

void ComponentFace::execute(BhIR *bhir) {
    BH_REQUIRE_INIT();
    _implementation->execute(bhir);
}
void ComponentFace::extmethod(const string &name, bh_opcode opcode) {
    BH_REQUIRE_INIT();
    _implementation->extmethod(name, opcode);
}
string ComponentFace::message(const string &msg) {
    if (!initiated()) return string(); // the end of the stack adds nothing
    return _implementation->message(msg);
}
void *ComponentFace::getMemoryPointer(bh_base &base, bool copy2host, bool force_alloc, bool nullify) {
    BH_REQUIRE_INIT();
    return _implementation->getMemoryPointer(base, copy2host, force_alloc, nullify);
}
void ComponentFace::setMemoryPointer(bh_base *base, bool host_ptr, void *mem) {
    BH_REQUIRE_INIT();
    _implementation->setMemoryPointer(base, host_ptr, mem);
}
void ComponentFace::memCopy(bh_view &src, bh_view &dst, const string &param) {
    BH_REQUIRE_INIT();
    _implementation->memCopy(src, dst, param);
}
void *ComponentFace::getDeviceContext() {
    if (!initiated()) return nullptr;
    return _implementation->getDeviceContext();
}
void ComponentFace::setDeviceContext(void *device_context) {
    if (!initiated()) return;
    _implementation->setDeviceContext(device_context);
}
string ComponentFace::userKernel(const string &kernel, vector<bh_view> &operand_list, const string &compile_cmd,
                                 const string &tag, const string &param) {
    BH_REQUIRE_INIT();
    return _implementation->userKernel(kernel, operand_list, compile_cmd, tag, param);
}

} // namespace component

// ---------------------------------------------------------------------------------------------
namespace extmethod {

ExtmethodFace::ExtmethodFace(const ConfigParser &parent_config, const string &name) : _name(name) {
    vector<string> libs;
    try {
        libs = parent_config.getListOfPaths("libs");
    } catch (const ConfigKeyNotFound &) {
    }
    const string fcreate = name + "_create";
    const string fdestroy = name + "_destroy";
    string err_msg;
    for (const string &lib_path : libs) {
        void *handle = dlopen(lib_path.c_str(), RTLD_NOW);
        if (handle == nullptr) throw runtime_error(string("Extmethod: cannot load library: ") + dlerror());
        dlerror();
        *reinterpret_cast<void **>(&_create) = dlsym(handle, fcreate.c_str());
        const bool has_create = dlerror() == nullptr;
        *reinterpret_cast<void **>(&_destroy) = dlsym(handle, fdestroy.c_str());
        const bool has_destroy = dlerror() == nullptr;
        if (has_create && has_destroy) {
            _lib_handle = handle;
            _implementation = _create();
            return;
        }
        err_msg += "'" + name + "' not in " + lib_path + "; ";
        dlclose(handle);
    }
    throw ExtmethodNotFound("Extmethod: cannot find '" + name + "': " + err_msg);
}

ExtmethodFace::~ExtmethodFace() {
    if (_implementation != nullptr) _destroy(_implementation);
}

} // namespace extmethod
} // namespace bohrium
