// gg_tune.cpp -- the autotuner's persistent cache.
//
// Tuned launch shapes (the single-graph engine's batch width, resident blocks and
// walk depth; the batched evaluator's chunk width per base; the lift evaluator's
// group size) are kept per process in a map and in a text file, so that a later
// process on the same kind of GPU starts from the tuned shape.  One line per
// entry:  <key> TAB <int> <int> ...   where the key names the GPU (device name and
// SM count), the evaluator and the problem shape.  The file is rewritten whole
// (temporary file renamed into place) after every new entry.
//
// File: GG_TUNE_CACHE if set ("off" or empty: no file), else
// $XDG_CACHE_HOME/graphgolf-b200/tune.tsv, else $HOME/.cache/graphgolf-b200/tune.tsv;
// gg_set_tune_cache() overrides both.
#include "gg.h"
#include "gg_internal.h"

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <unistd.h>
#include <vector>

namespace {

std::mutex g_mu;
std::map<std::string, std::vector<int>> g_map;
bool g_loaded = false;
bool g_path_set = false;
std::string g_path;

std::string default_path() {
    const char *env = std::getenv("GG_TUNE_CACHE");
    if (env) return (std::string(env) == "off") ? std::string() : std::string(env);
    const char *xdg = std::getenv("XDG_CACHE_HOME");
    const char *home = std::getenv("HOME");
    std::string dir;
    if (xdg && *xdg) dir = xdg;
    else if (home && *home) dir = std::string(home) + "/.cache";
    else return std::string();
    return dir + "/graphgolf-b200/tune.tsv";
}

const std::string &path_locked() {
    if (!g_path_set) {
        g_path = default_path();
        g_path_set = true;
    }
    return g_path;
}

void load_locked() {
    if (g_loaded) return;
    g_loaded = true;
    const std::string &p = path_locked();
    if (p.empty()) return;
    std::ifstream in(p);
    std::string line;
    while (std::getline(in, line)) {
        const auto tab = line.find('\t');
        if (tab == std::string::npos || tab == 0) continue;
        std::istringstream vs(line.substr(tab + 1));
        std::vector<int> v;
        int x;
        while (vs >> x) v.push_back(x);
        if (!v.empty()) g_map.emplace(line.substr(0, tab), v);  // entries made in this process win
    }
}

void mkdirs(const std::string &file) {
    for (size_t i = 1; i < file.size(); ++i)
        if (file[i] == '/') mkdir(file.substr(0, i).c_str(), 0755);
}

void save_locked() {
    const std::string &p = path_locked();
    if (p.empty()) return;
    mkdirs(p);
    const std::string tmp = p + ".tmp." + std::to_string((long long)getpid());
    {
        std::ofstream out(tmp, std::ios::trunc);
        if (!out) return;
        for (const auto &kv : g_map) {
            out << kv.first << '\t';
            for (size_t i = 0; i < kv.second.size(); ++i) out << (i ? " " : "") << kv.second[i];
            out << '\n';
        }
        if (!out) { std::remove(tmp.c_str()); return; }
    }
    if (std::rename(tmp.c_str(), p.c_str()) != 0) std::remove(tmp.c_str());
}

}  // namespace

namespace gg {

std::string tune_key(int device, const char *what, const std::vector<long long> &dims) {
    static std::mutex mu;
    static std::map<int, std::string> names;   // the device query is slow: once per device
    std::string gpu;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = names.find(device);
        if (it != names.end()) {
            gpu = it->second;
        } else {
            cudaDeviceProp prop{};
            gpu = "unknown";
            if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) {
                gpu = prop.name;
                gpu += "/" + std::to_string(prop.multiProcessorCount) + "sm";
            } else {
                (void)cudaGetLastError();
            }
            for (auto &c : gpu)
                if (c == '\t' || c == '\n' || c == '|') c = ' ';
            names[device] = gpu;
        }
    }
    // the format version also retires entries tuned for earlier kernels (v2: the
    // level kernel at 4 resident blocks a SM, the walk of all batches in one launch)
    std::string k = "v2|" + gpu + "|" + what;
    for (long long d : dims) k += "|" + std::to_string(d);
    return k;
}

bool tune_get(const std::string &key, std::vector<int> *vals) {
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    auto it = g_map.find(key);
    if (it == g_map.end()) return false;
    *vals = it->second;
    return true;
}

void tune_put(const std::string &key, const std::vector<int> &vals) {
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    g_map[key] = vals;
    save_locked();
}

}  // namespace gg

extern "C" gg_status gg_set_tune_cache(const char *path) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_path = path ? std::string(path) : std::string();
    g_path_set = true;
    g_loaded = false;   // entries of the new file are read on the next lookup
    return GG_OK;
}
