// The autotuner's choice cache as a JSON file: one flat object whose keys name the choice, the
// device and the workload shape, and whose values are the choice (a probe batch, a tile shape).
//
//   {"batch|NVIDIA B200/148|1024,1024,2,256": 256, "tile|NVIDIA B200/148|512,512,1": 1}
//
// Entries of other devices stay in the file untouched; a file that cannot be read or parsed is
// treated as empty.  Writes go to a temporary file renamed over the old one.
#include <cuda_runtime.h>

#include <cctype>
#include <exception>
#include <cstdio>
#include <fstream>
#include <map>
#include <sstream>
#include <string>

#include "ctx.hpp"

namespace msb {

namespace {
// every "key": integer pair of a flat JSON object (keys hold no quotes or backslashes)
std::map<std::string, long> parse_flat(const std::string& text)
{
    std::map<std::string, long> out;
    size_t i = 0;
    const size_t n = text.size();
    while (i < n) {
        const size_t q0 = text.find('"', i);
        if (q0 == std::string::npos) break;
        const size_t q1 = text.find('"', q0 + 1);
        if (q1 == std::string::npos) break;
        std::string key = text.substr(q0 + 1, q1 - q0 - 1);
        size_t j = q1 + 1;
        while (j < n && std::isspace((unsigned char)text[j])) j++;
        if (j >= n || text[j] != ':') {
            i = q1 + 1;
            continue;
        }
        j++;
        while (j < n && std::isspace((unsigned char)text[j])) j++;
        size_t k = j;
        if (k < n && (text[k] == '-' || text[k] == '+')) k++;
        while (k < n && std::isdigit((unsigned char)text[k])) k++;
        if (k > j && std::isdigit((unsigned char)text[k - 1])) {
            try {
                out[key] = std::stol(text.substr(j, k - j));
            } catch (const std::exception&) {
                // a value out of range: the entry is dropped
            }
        }
        i = k > j ? k : j + 1;
    }
    return out;
}

std::map<std::string, long> read_file(const std::string& path)
{
    std::ifstream f(path);
    if (!f) return {};
    std::stringstream ss;
    ss << f.rdbuf();
    return parse_flat(ss.str());
}
}  // namespace

std::string device_tag(ms_ctx* c)
{
    if (c->device_tag.empty()) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, c->device) == cudaSuccess)
            c->device_tag = std::string(prop.name) + "/" + std::to_string(prop.multiProcessorCount);
        else
            c->device_tag = "device" + std::to_string(c->device);
    }
    return c->device_tag;
}

void tune_load(ms_ctx* c)
{
    if (c->tune_path.empty()) return;
    const std::string tag = device_tag(c);
    for (const auto& kv : read_file(c->tune_path)) {
        const std::string& k = kv.first;
        const size_t a = k.find('|'), b = a == std::string::npos ? a : k.find('|', a + 1);
        if (b == std::string::npos || k.compare(a + 1, b - a - 1, tag) != 0) continue;
        const std::string kind = k.substr(0, a), rest = k.substr(b + 1);
        // values outside the choices the tuner makes are dropped (an edited or damaged file)
        if (kind == "batch" && kv.second >= 1 && kv.second <= 256) c->batch_choice[rest] = (int)kv.second;
        else if (kind == "tile" && kv.second >= 0 && kv.second <= 7) c->tile_choice[rest] = (int)kv.second;
    }
}

void tune_save(ms_ctx* c)
{
    if (c->tune_path.empty()) return;
    const std::string tag = device_tag(c);
    std::map<std::string, long> all = read_file(c->tune_path);   // keeps other devices' entries
    for (const auto& kv : c->batch_choice) all["batch|" + tag + "|" + kv.first] = kv.second;
    for (const auto& kv : c->tile_choice) all["tile|" + tag + "|" + kv.first] = kv.second;
    const std::string tmp = c->tune_path + ".tmp";
    {
        std::ofstream f(tmp, std::ios::trunc);
        if (!f) return;   // an unwritable cache only loses the persistence
        f << "{";
        bool first = true;
        for (const auto& kv : all) {
            f << (first ? "\n  " : ",\n  ") << '"' << kv.first << "\": " << kv.second;
            first = false;
        }
        f << "\n}\n";
        if (!f) return;
    }
    std::rename(tmp.c_str(), c->tune_path.c_str());
}

}  // namespace msb
