// config.txt parser: the host side of the boundary's configuration.
//
// Restates GameConfigData::setConfigDataFromFile / getInt / getFloat
// (game_configdata.cpp:22-90) and the key reads of
// Simulation::initDeviceParams (Simulation.cpp:56-77) without process-global
// state and without exit(1): every failure becomes MPM_ERR_BAD_CONFIG.
//
// Format rules kept from the reference because they change what a file means:
//  - every ' ' is removed from a line before anything else (line 28), so
//    "SIZE_X = 1 28" reads as 128; tabs and '\r' are kept;
//  - a line is split at its first '='; lines without '=' are ignored;
//  - WATER=/OBJECT= values are split on ';' like std::getline does (a
//    trailing empty field is dropped) and need >= 5 fields (lines 35-49);
//  - integers parse like std::stoi: optional leading whitespace and sign, then
//    the longest digit prefix ("0.5" -> 0, "12abc" -> 12); no digits or an
//    out-of-range value is an error;
//  - floats parse like std::stof (strtof): prefix parse, ERANGE is an error.
#include "mpm_b200.h"

#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

struct Entry {
    std::string path;
    float scale, x, y, z;
};

struct Parsed {
    std::unordered_map<std::string, std::string> kv;
    std::vector<Entry> waters, objects;
};

// std::stoi semantics (strtol + int range check).
bool parse_int(const std::string& s, int32_t* out) {
    const char* b = s.c_str();
    char* e = nullptr;
    errno = 0;
    long v = std::strtol(b, &e, 10);
    if (e == b) return false;
    if (errno == ERANGE || v < INT_MIN || v > INT_MAX) return false;
    *out = (int32_t)v;
    return true;
}

// std::stof semantics (strtof; ERANGE raises in std::stof).
bool parse_float(const std::string& s, float* out) {
    const char* b = s.c_str();
    char* e = nullptr;
    errno = 0;
    float v = std::strtof(b, &e);
    if (e == b) return false;
    if (errno == ERANGE) return false;
    *out = v;
    return true;
}

// std::getline-based split (game_configdata.cpp:8-17).
std::vector<std::string> split(const std::string& s, char d) {
    std::vector<std::string> parts;
    std::string tok;
    std::istringstream is(s);
    while (std::getline(is, tok, d)) parts.push_back(tok);
    return parts;
}

bool parse_text(std::istream& in, Parsed& p, std::string& err) {
    std::string line;
    while (std::getline(in, line)) {
        std::string l;
        l.reserve(line.size());
        for (char c : line)
            if (c != ' ') l.push_back(c);
        if (l.empty()) continue;
        size_t eq = l.find('=');
        if (eq == std::string::npos) continue;
        std::string key = l.substr(0, eq), value = l.substr(eq + 1);
        if (key == "WATER" || key == "OBJECT") {
            std::vector<std::string> parts = split(value, ';');
            if (parts.size() < 5) {
                err = "malformed " + key + " entry '" + value + "': expected path;scale;x;y;z";
                return false;
            }
            Entry en;
            en.path = parts[0];
            float* dst[4] = {&en.scale, &en.x, &en.y, &en.z};
            for (int i = 0; i < 4; ++i) {
                if (!parse_float(parts[1 + i], dst[i])) {
                    err = "malformed " + key + " entry '" + value + "': field " + std::to_string(i + 2) +
                          " is not a float";
                    return false;
                }
            }
            (key == "WATER" ? p.waters : p.objects).push_back(en);
        } else {
            p.kv[key] = value;
        }
    }
    return true;
}

bool get_int(const Parsed& p, const char* key, int32_t* out, std::string& err) {
    auto it = p.kv.find(key);
    if (it == p.kv.end()) {
        err = std::string("missing key ") + key;
        return false;
    }
    if (!parse_int(it->second, out)) {
        err = std::string("key ") + key + " is not an integer: '" + it->second + "'";
        return false;
    }
    return true;
}

bool get_float(const Parsed& p, const char* key, float* out, std::string& err) {
    auto it = p.kv.find(key);
    if (it == p.kv.end()) {
        err = std::string("missing key ") + key;
        return false;
    }
    if (!parse_float(it->second, out)) {
        err = std::string("key ") + key + " is not a float: '" + it->second + "'";
        return false;
    }
    return true;
}

void put_err(char* err, int32_t err_len, const std::string& msg) {
    if (!err || err_len <= 0) return;
    size_t n = std::min((size_t)(err_len - 1), msg.size());
    std::memcpy(err, msg.data(), n);
    err[n] = '\0';
}

void copy_entries(const std::vector<Entry>& src, mpm_scene_entry* dst, int32_t max, int32_t* count) {
    if (count) *count = (int32_t)src.size();
    if (!dst) return;
    for (int32_t i = 0; i < max && i < (int32_t)src.size(); ++i) {
        std::memset(&dst[i], 0, sizeof(mpm_scene_entry));
        std::strncpy(dst[i].model_path, src[i].path.c_str(), MPM_PATH_MAX - 1);
        dst[i].scale = src[i].scale;
        dst[i].x = src[i].x;
        dst[i].y = src[i].y;
        dst[i].z = src[i].z;
    }
}

mpm_status finish(std::istream& in, mpm_config* cfg, mpm_scene_entry* waters, int32_t max_waters,
                  int32_t* n_waters, mpm_scene_entry* objects, int32_t max_objects, int32_t* n_objects,
                  char* err, int32_t err_len) {
    Parsed p;
    std::string e;
    if (!parse_text(in, p, e)) {
        put_err(err, err_len, e);
        return MPM_ERR_BAD_CONFIG;
    }
    mpm_config c;
    std::memset(&c, 0, sizeof(c));
    // Read order of Simulation::initDeviceParams (Simulation.cpp:59-69).
    bool ok = get_int(p, "SIZE_X", &c.size_x, e) && get_int(p, "SIZE_Y", &c.size_y, e) &&
              get_int(p, "SIZE_Z", &c.size_z, e) && get_int(p, "PADDING", &c.padding, e) &&
              get_float(p, "GRAVITY", &c.gravity, e) && get_float(p, "DT", &c.dt, e) &&
              get_float(p, "GAMMA", &c.gamma, e) && get_float(p, "COMPRESSION", &c.compression, e) &&
              get_float(p, "RESOLUTION", &c.resolution, e) && get_int(p, "SUBSTEPS", &c.substeps, e) &&
              get_int(p, "SDF_RESOLUTION", &c.sdf_resolution, e);
    if (!ok) {
        put_err(err, err_len, e);
        return MPM_ERR_BAD_CONFIG;
    }
    if (cfg) *cfg = c;
    copy_entries(p.waters, waters, max_waters, n_waters);
    copy_entries(p.objects, objects, max_objects, n_objects);
    put_err(err, err_len, "");
    return MPM_OK;
}

}  // namespace

extern "C" mpm_status mpm_config_parse_string(const char* text, mpm_config* cfg, mpm_scene_entry* waters,
                                              int32_t max_waters, int32_t* n_waters, mpm_scene_entry* objects,
                                              int32_t max_objects, int32_t* n_objects, char* err,
                                              int32_t err_len) {
    if (!text) {
        put_err(err, err_len, "text is NULL");
        return MPM_ERR_INVALID_ARGUMENT;
    }
    std::istringstream in{std::string(text)};
    return finish(in, cfg, waters, max_waters, n_waters, objects, max_objects, n_objects, err, err_len);
}

extern "C" mpm_status mpm_config_parse_file(const char* path, mpm_config* cfg, mpm_scene_entry* waters,
                                            int32_t max_waters, int32_t* n_waters, mpm_scene_entry* objects,
                                            int32_t max_objects, int32_t* n_objects, char* err,
                                            int32_t err_len) {
    if (!path) {
        put_err(err, err_len, "path is NULL");
        return MPM_ERR_INVALID_ARGUMENT;
    }
    std::ifstream in(path);
    if (!in.is_open()) {
        put_err(err, err_len, std::string("cannot open config file ") + path);
        return MPM_ERR_IO;
    }
    return finish(in, cfg, waters, max_waters, n_waters, objects, max_objects, n_objects, err, err_len);
}

namespace mpm {
// `key` of a config text read as GameConfigData::getInt reads it (std::stoi of
// the space-stripped value): the scene builder's lattice step is
// getInt("RESOLUTION") (VoxelEngine.cpp:369), not the float the kernels use.
bool config_text_int(const char* text, const char* key, int32_t* out, std::string& err) {
    std::istringstream in(text ? text : "");
    Parsed p;
    if (!parse_text(in, p, err)) return false;
    return get_int(p, key, out, err);
}
}  // namespace mpm
