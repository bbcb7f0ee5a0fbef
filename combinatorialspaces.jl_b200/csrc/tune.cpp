// The autotuner's table (tune.cuh).
#include "tune.cuh"

#include <cuda_runtime.h>

#include <atomic>
#include <cctype>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

#include "common.cuh"

namespace decb {
namespace {
std::mutex g_mu;
std::atomic<unsigned> g_version{1};
std::map<std::string, int>& table() {
  static std::map<std::string, int> t;
  return t;
}
}  // namespace

int size_bucket(long long n) {
  int b = 0;
  while (n > 1) {
    n >>= 1;
    ++b;
  }
  return b;
}

int tune_get(const std::string& key, int dflt) {
  std::lock_guard<std::mutex> lock(g_mu);
  auto it = table().find(key);
  return it == table().end() ? dflt : it->second;
}

void tune_set(const std::string& key, int value) {
  std::lock_guard<std::mutex> lock(g_mu);
  table()[key] = value;
  g_version.fetch_add(1);
}

unsigned tune_version() { return g_version.load(); }

void tune_clear() {
  std::lock_guard<std::mutex> lock(g_mu);
  table().clear();
  g_version.fetch_add(1);
}

void tune_save(const std::string& path) {
  std::string device = "unknown";
  int dev = 0;
  cudaDeviceProp prop;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess) device = prop.name;
  else (void)cudaGetLastError();
  std::ostringstream os;
  os << "{\n \"format\": \"dec_b200 tuning table\",\n \"version\": 1,\n \"device\": \"" << device
     << "\",\n \"entries\": {";
  {
    std::lock_guard<std::mutex> lock(g_mu);
    bool first = true;
    for (const auto& kv : table()) {
      os << (first ? "\n  \"" : ",\n  \"") << kv.first << "\": " << kv.second;
      first = false;
    }
  }
  os << "\n }\n}\n";
  std::ofstream f(path);
  require(f.good(), "tuning table: cannot open the file for writing");
  f << os.str();
  require(f.good(), "tuning table: write failed");
}

int tune_load(const std::string& path) {
  std::ifstream f(path);
  require(f.good(), "tuning table: cannot open the file");
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string s = ss.str();
  require(s.find("\"dec_b200 tuning table\"") != std::string::npos, "tuning table: not a dec_b200 tuning table");
  size_t p = s.find("\"entries\"");
  require(p != std::string::npos, "tuning table: no entries");
  p = s.find('{', p);
  require(p != std::string::npos, "tuning table: malformed entries");
  const size_t end = s.find('}', p);
  require(end != std::string::npos, "tuning table: malformed entries");
  std::map<std::string, int> read;
  size_t q = p + 1;
  while (true) {
    const size_t k0 = s.find('"', q);
    if (k0 == std::string::npos || k0 > end) break;
    const size_t k1 = s.find('"', k0 + 1);
    require(k1 != std::string::npos && k1 < end, "tuning table: malformed key");
    const std::string key = s.substr(k0 + 1, k1 - k0 - 1);
    for (char c : key)
      require(std::isalnum((unsigned char)c) || c == '/' || c == '_' || c == '.' || c == '-',
              "tuning table: bad character in a key");
    size_t c = s.find(':', k1);
    require(c != std::string::npos && c < end, "tuning table: malformed entry");
    ++c;
    while (c < end && std::isspace((unsigned char)s[c])) ++c;
    size_t v1 = c;
    if (v1 < end && s[v1] == '-') ++v1;
    while (v1 < end && std::isdigit((unsigned char)s[v1])) ++v1;
    require(v1 > c, "tuning table: entry value must be an integer");
    read[key] = std::stoi(s.substr(c, v1 - c));
    q = v1;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  for (const auto& kv : read) table()[kv.first] = kv.second;
  g_version.fetch_add(1);
  return (int)read.size();
}
}  // namespace decb
