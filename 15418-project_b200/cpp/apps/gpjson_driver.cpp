// gpjson_driver: runs JSONPath queries over a JSON-lines file with the B200
// engine.  Same configuration surface as the reference's driver
// (apps/driver_config.cpp:266-359, apps/main.cpp): TOML keys
//   run_name, dataset_path, queries,
//   [file_reader] type, [index_builder] type / file_partition_size /
//   grid_size / block_size / reduction_grid_size / reduction_block_size,
//   [query_executor] grid_size / block_size
// and the matching command-line options (--dataset-path, alias --dataset;
// --queries, aliases --query and -q; --index-builder.grid-size, ...), with
// the command line overriding the file.  Prints the same "### RUN BEGIN",
// "GPJSON_RUN_CONFIG {json}", profiler and summary lines.
#include "gpjson/engine.hpp"
#include "gpjson/error/error.hpp"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

struct Inputs {
  std::string run_name;
  std::string dataset_path;
  std::vector<std::string> queries;
  gpjson::EngineOptions options;
};

// ---- a small TOML subset: [tables], key = "string" | integer | ["a", ...] --
struct TomlValue {
  enum Kind { kString, kInt, kArray } kind = kString;
  std::string s;
  int64_t i = 0;
  std::vector<std::string> arr;
};

std::string parse_toml_string(const std::string &line, size_t &p) {
  const char q = line[p++];
  std::string out;
  while (p < line.size() && line[p] != q) {
    char c = line[p++];
    if (q == '"' && c == '\\' && p < line.size()) {
      const char e = line[p++];
      switch (e) {
        case 'n': c = '\n'; break;
        case 't': c = '\t'; break;
        case 'r': c = '\r'; break;
        case '"': c = '"'; break;
        case '\\': c = '\\'; break;
        default: out.push_back('\\'); c = e; break;
      }
    }
    out.push_back(c);
  }
  if (p >= line.size()) throw std::runtime_error("TOML: unterminated string");
  ++p;
  return out;
}

void skip_ws(const std::string &s, size_t &p) {
  while (p < s.size() && (s[p] == ' ' || s[p] == '\t')) ++p;
}

std::map<std::string, TomlValue> parse_toml(const std::string &path) {
  std::ifstream in(path);
  if (!in) throw std::runtime_error("cannot open config file '" + path + "'");
  std::map<std::string, TomlValue> out;
  std::string table, line, pending;
  while (std::getline(in, line)) {
    if (!pending.empty()) {  // multi-line array
      pending += " " + line;
      if (line.find(']') == std::string::npos) continue;
      line = pending;
      pending.clear();
    }
    size_t p = 0;
    skip_ws(line, p);
    if (p >= line.size() || line[p] == '#') continue;
    if (line[p] == '[') {
      const size_t e = line.find(']', p);
      if (e == std::string::npos) throw std::runtime_error("TOML: bad table header");
      table = line.substr(p + 1, e - p - 1);
      continue;
    }
    const size_t eq = line.find('=', p);
    if (eq == std::string::npos) throw std::runtime_error("TOML: expected key = value");
    std::string key = line.substr(p, eq - p);
    while (!key.empty() && (key.back() == ' ' || key.back() == '\t')) key.pop_back();
    size_t v = eq + 1;
    skip_ws(line, v);
    if (v < line.size() && line[v] == '[' && line.find(']', v) == std::string::npos) {
      pending = line;
      continue;
    }
    TomlValue val;
    if (v < line.size() && (line[v] == '"' || line[v] == '\'')) {
      val.kind = TomlValue::kString;
      val.s = parse_toml_string(line, v);
    } else if (v < line.size() && line[v] == '[') {
      val.kind = TomlValue::kArray;
      ++v;
      for (;;) {
        skip_ws(line, v);
        if (v < line.size() && line[v] == ']') break;
        if (v >= line.size() || (line[v] != '"' && line[v] != '\''))
          throw std::runtime_error("TOML array '" + key + "' must contain only strings.");
        val.arr.push_back(parse_toml_string(line, v));
        skip_ws(line, v);
        if (v < line.size() && line[v] == ',') ++v;
      }
    } else {
      size_t e = v;
      while (e < line.size() && line[e] != '#' && line[e] != ' ') ++e;
      const std::string num = line.substr(v, e - v);
      try {
        size_t used = 0;
        val.i = std::stoll(num, &used);
        if (used != num.size()) throw std::invalid_argument(num);
        val.kind = TomlValue::kInt;
      } catch (const std::exception &) {
        throw std::runtime_error("TOML value for '" + key + "' has the wrong type.");
      }
    }
    out[table.empty() ? key : table + "." + key] = val;
  }
  return out;
}

gpjson::file::FileReaderType reader_type(const std::string &t) {
  if (t == "COPIED") return gpjson::file::FileReaderType::COPIED;
  if (t == "MMAP") return gpjson::file::FileReaderType::MMAP;
  throw std::runtime_error("Invalid enum value '" + t + "'. Expected one of: COPIED, MMAP");
}

gpjson::index::IndexBuilderType builder_type(const std::string &t) {
  using T = gpjson::index::IndexBuilderType;
  if (t == "UNCOMBINED") return T::UNCOMBINED;
  if (t == "COMBINED") return T::COMBINED;
  if (t == "FUSED") return T::FUSED;
  if (t == "SHAREMEM") return T::SHAREMEM;
  if (t == "B200") return T::B200;
  throw std::runtime_error("Invalid enum value '" + t +
                           "'. Expected one of: UNCOMBINED, COMBINED, FUSED, SHAREMEM, B200");
}

template <class T>
T narrow(int64_t v, const std::string &key) {
  if (v < int64_t(std::numeric_limits<T>::lowest()) ||
      (v > 0 && uint64_t(v) > uint64_t(std::numeric_limits<T>::max())) ||
      (std::is_unsigned<T>::value && v < 0))
    throw std::runtime_error("TOML value for '" + key + "' is out of range.");
  return T(v);
}

// Applies one setting (from TOML or the command line) to the inputs.
void apply(Inputs &in, const std::string &key, const TomlValue &v) {
  auto need_int = [&]() {
    if (v.kind != TomlValue::kInt)
      throw std::runtime_error("TOML value for '" + key + "' must be an integer.");
    return v.i;
  };
  auto need_str = [&]() {
    if (v.kind != TomlValue::kString)
      throw std::runtime_error("TOML value for '" + key + "' has the wrong type.");
    return v.s;
  };
  auto &ib = in.options.index_builder_options;
  auto &qe = in.options.query_executor_options;
  if (key == "run_name") in.run_name = need_str();
  else if (key == "dataset_path") in.dataset_path = need_str();
  else if (key == "queries") {
    if (v.kind != TomlValue::kArray)
      throw std::runtime_error("TOML value for 'queries' must be an array of strings.");
    in.queries = v.arr;
  } else if (key == "file_reader.type") in.options.file_reader_options.file_reader_type = reader_type(need_str());
  else if (key == "index_builder.type") ib.index_builder_type = builder_type(need_str());
  else if (key == "index_builder.file_partition_size") ib.file_partition_size = narrow<size_t>(need_int(), key);
  else if (key == "index_builder.grid_size") ib.grid_size = narrow<int>(need_int(), key);
  else if (key == "index_builder.block_size") ib.block_size = narrow<int>(need_int(), key);
  else if (key == "index_builder.reduction_grid_size") ib.reduction_grid_size = narrow<int>(need_int(), key);
  else if (key == "index_builder.reduction_block_size") ib.reduction_block_size = narrow<int>(need_int(), key);
  else if (key == "query_executor.grid_size") qe.grid_size = narrow<int>(need_int(), key);
  else if (key == "query_executor.block_size") qe.block_size = narrow<int>(need_int(), key);
}

// Command-line names: "--" + key with '_' -> '-', plus the aliases.
std::string key_of_option(const std::string &opt) {
  static const std::map<std::string, std::string> kAlias = {
      {"--dataset", "dataset_path"}, {"--query", "queries"}, {"-q", "queries"}};
  auto it = kAlias.find(opt);
  if (it != kAlias.end()) return it->second;
  if (opt.rfind("--", 0) != 0) return "";
  std::string k = opt.substr(2);
  for (char &c : k)
    if (c == '-') c = '_';
  return k;
}

bool is_int_key(const std::string &k) {
  return k.find("size") != std::string::npos;
}

std::string json_escape(const std::string &s) {
  std::ostringstream o;
  for (unsigned char c : s) {
    switch (c) {
      case '"': o << "\\\""; break;
      case '\\': o << "\\\\"; break;
      case '\n': o << "\\n"; break;
      case '\t': o << "\\t"; break;
      case '\r': o << "\\r"; break;
      case '\b': o << "\\b"; break;
      case '\f': o << "\\f"; break;
      default:
        if (c < 0x20) o << "\\u" << std::hex << std::setw(4) << std::setfill('0') << int(c) << std::dec;
        else o << char(c);
    }
  }
  return o.str();
}

std::string config_json(const Inputs &in) {
  std::ostringstream o;
  const auto &ib = in.options.index_builder_options;
  const auto &qe = in.options.query_executor_options;
  std::ostringstream rt, bt;
  rt << in.options.file_reader_options.file_reader_type;
  bt << ib.index_builder_type;
  o << "{\"run_name\":\"" << json_escape(in.run_name) << "\",\"dataset_path\":\""
    << json_escape(in.dataset_path) << "\",\"queries\":[";
  for (size_t i = 0; i < in.queries.size(); ++i)
    o << (i ? "," : "") << "\"" << json_escape(in.queries[i]) << "\"";
  o << "],\"engine_options\":{\"file_reader\":{\"type\":\"" << rt.str()
    << "\"},\"index_builder\":{\"type\":\"" << bt.str()
    << "\",\"file_partition_size\":" << ib.file_partition_size
    << ",\"grid_size\":" << ib.grid_size << ",\"block_size\":" << ib.block_size
    << ",\"reduction_grid_size\":" << ib.reduction_grid_size
    << ",\"reduction_block_size\":" << ib.reduction_block_size
    << "},\"query_executor\":{\"grid_size\":" << qe.grid_size
    << ",\"block_size\":" << qe.block_size << "}}}";
  return o.str();
}

Inputs parse_inputs(int argc, char **argv) {
  Inputs in;
  in.run_name = "run_" + std::to_string(std::chrono::duration_cast<std::chrono::milliseconds>(
                                            std::chrono::system_clock::now().time_since_epoch())
                                            .count());
  std::vector<std::string> args(argv + 1, argv + argc);
  for (size_t i = 0; i < args.size(); ++i) {  // the config file first
    if ((args[i] == "-c" || args[i] == "--config") && i + 1 < args.size()) {
      for (auto &kv : parse_toml(args[i + 1])) apply(in, kv.first, kv.second);
    }
  }
  std::vector<std::string> cli_queries;
  bool cli_has_queries = false;
  for (size_t i = 0; i < args.size(); ++i) {
    const std::string &a = args[i];
    if (a == "-c" || a == "--config") {
      ++i;
      continue;
    }
    if (a == "-h" || a == "--help") {
      std::cout << "Usage: gpjson_driver [-c CONFIG.toml] [--dataset PATH] [-q QUERY ...]\n"
                   "  [--run-name N] [--file-reader.type COPIED|MMAP]\n"
                   "  [--index-builder.type T] [--index-builder.file-partition-size N]\n"
                   "  [--query-executor.grid-size N] [--query-executor.block-size N]\n";
      std::exit(0);
    }
    const std::string key = key_of_option(a);
    if (key.empty() || i + 1 >= args.size())
      throw std::runtime_error("The following argument was not expected: " + a);
    if (key == "queries") {
      cli_has_queries = true;
      while (i + 1 < args.size() && args[i + 1].rfind("-", 0) != 0) cli_queries.push_back(args[++i]);
      continue;
    }
    TomlValue v;
    const std::string val = args[++i];
    if (is_int_key(key)) {
      v.kind = TomlValue::kInt;
      try {
        v.i = std::stoll(val);
      } catch (const std::exception &) {
        throw std::runtime_error(a + ": Value " + val + " could not be converted");
      }
    } else {
      v.s = val;
    }
    apply(in, key, v);
  }
  if (cli_has_queries) in.queries = cli_queries;
  if (in.run_name.empty()) throw std::runtime_error("run_name must not be empty.");
  if (in.dataset_path.empty())
    throw std::runtime_error(
        "dataset_path is required. Use --dataset or set dataset_path in the TOML config.");
  if (in.queries.empty())
    throw std::runtime_error("At least one query is required. Use --query or set queries in the TOML config.");
  const auto &ib = in.options.index_builder_options;
  const auto &qe = in.options.query_executor_options;
  if (ib.grid_size < 0 || ib.block_size < 0 || ib.reduction_grid_size < 0 ||
      ib.reduction_block_size < 0)
    throw std::runtime_error("Index builder grid and block sizes must be non-negative.");
  if (qe.grid_size < 0 || qe.block_size < 0)
    throw std::runtime_error("Query executor grid and block sizes must be non-negative.");
  return in;
}

}  // namespace

int main(int argc, char **argv) {
  try {
    const Inputs in = parse_inputs(argc, argv);
    std::cout << "### RUN BEGIN run_name=" << in.run_name << " ###\n";
    std::cout << "GPJSON_RUN_CONFIG " << config_json(in) << "\n" << std::flush;
    gpjson::Engine engine;
    const auto result = engine.query(in.dataset_path, in.queries, in.options);
    std::cout << "Result has " << result.queries().size() << " queries\n";
    for (const auto &q : result.queries()) {
      unsigned long matches = 0;
      for (const auto &line : q.lines()) matches += line.values().size();
      std::cout << "Query '" << q.query_text() << "' has " << q.lines().size()
                << " lines of result, and " << matches << " matched values\n";
    }
    std::cout << "### RUN END run_name=" << in.run_name << " ###\n";
    return 0;
  } catch (const std::exception &e) {
    std::cerr << "gpjson_driver: " << e.what() << '\n';
    return 1;
  }
}
