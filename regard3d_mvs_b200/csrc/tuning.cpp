// Reads the autotuner's launch-shape table (tuning.h).
#include "tuning.h"

#include <dlfcn.h>

#include <cstdlib>
#include <fstream>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>

namespace r3dgpu {
namespace {

std::string default_path() {
  Dl_info info{};
  if (dladdr(reinterpret_cast<void*>(&tuning), &info) == 0 || info.dli_fname == nullptr) return {};
  std::string lib(info.dli_fname);
  const size_t slash = lib.rfind('/');
  if (slash == std::string::npos) return {};
  const std::string dir = lib.substr(0, slash);         // .../regard3d_mvs_b200/_lib
  const size_t up = dir.rfind('/');
  return (up == std::string::npos ? std::string(".") : dir.substr(0, up)) + "/tuning_b200.txt";
}

Tuning parse(std::istream& in) {
  Tuning t;
  std::string line;
  while (std::getline(in, line)) {
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line.resize(hash);
    std::istringstream ss(line);
    std::string kind;
    if (!(ss >> kind)) continue;
    if (kind == "full") {
      int nd = 0, g = 0, k = 0, rows = 0;
      if (ss >> nd >> g >> k >> rows && nd > 0 && g > 0 && k > 0 && rows > 0) t.full[nd] = TunedFull{g, k, rows};
    } else if (kind == "ranged") {
      int width = 0, rows = 0;
      if (ss >> width >> rows && width > 0 && rows > 0) t.ranged_rows[width] = rows;
    } else if (kind == "ranged_wide_frac") {
      double f = -1.0;
      if (ss >> f && f >= 0.0) t.ranged_wide_frac = f;
    } else if (kind == "path") {
      int nd = 0, g = 0, k = 0;
      if (ss >> nd >> g >> k && nd > 0 && g > 0 && k > 0) t.path[nd] = TunedPath{g, k};
    } else if (kind == "ranged_general_width") {
      int w = 0;
      if (ss >> w && w > 0) t.ranged_general_width = w;
    }
  }
  t.loaded = true;
  return t;
}

Tuning load_file() {
  const char* env = std::getenv("R3DGPU_TUNING_FILE");
  const std::string path = env != nullptr ? std::string(env) : default_path();
  std::ifstream in(path);
  if (path.empty() || !in) return Tuning{};
  return parse(in);
}

}  // namespace

const Tuning& tuning() {
  // $R3DGPU_TUNING (the table's text, entries separated by newlines or ';')
  // is re-read whenever it changes, so that a tuning run can try tables in
  // one process; otherwise the file, read once.
  static const Tuning from_file = load_file();
  const char* env = std::getenv("R3DGPU_TUNING");
  if (env == nullptr) return from_file;
  static std::mutex mu;
  static std::string text;
  static std::shared_ptr<const Tuning> table;
  thread_local std::shared_ptr<const Tuning> held;  // keeps the returned table alive for this thread
  std::lock_guard<std::mutex> lk(mu);
  if (!table || text != env) {
    text = env;
    std::string lines = text;
    for (char& c : lines)
      if (c == ';') c = '\n';
    std::istringstream in(lines);
    table = std::make_shared<const Tuning>(parse(in));
  }
  held = table;
  return *held;
}

}  // namespace r3dgpu
