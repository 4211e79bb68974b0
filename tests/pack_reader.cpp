// Test helper: decodes a result pack written by sqsgenerator_b200.io with nlohmann::json::from_msgpack
// and reads it with the keys and value types that the reference's loader reads
// (adl_serializer<sqs_result_pack>::from_json and the serializers it calls, include/sqsgen/io/json.h:
// statistics :120-137, structure_config :160-174, configuration :176-212, interact/split results
// :214-238 with binary_adapter :33-50 for the SRO cube, pack :264-287; enums by name :289-310; maps with
// non-string keys as [key, value] arrays). Standard containers stand in for the Eigen types: a lattice
// or coordinate matrix as nested vectors, a cube as [S][K][K] vectors, the SRO tensor as shape + data.
// Prints a short summary; any missing key or wrong type throws (exit code 1).
//
// Usage: pack_reader <file> <single|double>
#include <array>
#include <cstdint>
#include <fstream>
#include <iostream>
#include <iterator>
#include <map>
#include <optional>
#include <set>
#include <string>
#include <vector>

#include <nlohmann/json.hpp>

using nlohmann::json;

// std::optional reads null as empty, as the reference's own serializer does (io/json.h:53-70).
NLOHMANN_JSON_NAMESPACE_BEGIN
template <class T> struct adl_serializer<std::optional<T>> {
  static void from_json(const json& j, std::optional<T>& o) {
    if (j.is_null())
      o = std::nullopt;
    else
      o = j.get<T>();
  }
};
NLOHMANN_JSON_NAMESPACE_END

template <class T> static std::optional<T> opt(const json& j) { return j.get<std::optional<T>>(); }

static void need_enum(const json& j, std::set<std::string> names) {
  if (!names.count(j.get<std::string>())) throw std::runtime_error("bad enum value " + j.dump());
}

template <class T> struct Reader {
  size_t results = 0, sro_values = 0;
  void config(const json& c) {
    need_enum(c.at("sublattice_mode"), {"interact", "split"});
    need_enum(c.at("iteration_mode"), {"random", "systematic"});
    auto seed = c.at("seed").get<std::vector<std::optional<uint64_t>>>();
    const json& s = c.at("structure");
    auto species = s.at("species").get<std::vector<uint8_t>>();
    auto lattice = s.at("lattice").get<std::vector<std::vector<T>>>();
    auto coords = s.at("coords").get<std::vector<std::vector<T>>>();
    auto supercell = s.at("supercell").get<std::array<size_t, 3>>();
    if (lattice.size() != 3 || coords.size() != species.size()) throw std::runtime_error("structure shape");
    for (const json& sl : c.at("composition")) {  // NLOHMANN_DEFINE_TYPE_NON_INTRUSIVE(sublattice, sites, composition)
      auto sites = sl.at("sites").get<std::set<size_t>>();
      auto comp = sl.at("composition").get<std::map<uint8_t, size_t>>();
      if (sites.empty() || comp.empty()) throw std::runtime_error("empty sublattice");
    }
    auto radii = c.at("shell_radii").get<std::vector<std::vector<T>>>();
    auto weights = c.at("shell_weights").get<std::vector<std::map<size_t, T>>>();
    for (const char* key : {"prefactors", "pair_weights", "target_objective"})
      auto cubes = c.at(key).get<std::vector<std::vector<std::vector<std::vector<T>>>>>();
    auto iterations = opt<uint64_t>(c.at("iterations"));
    auto chunk = c.at("chunk_size").get<uint64_t>();
    auto threads = c.at("thread_config").get<std::vector<size_t>>();
    auto keep = c.at("keep").get<size_t>();
    auto mrpo = opt<size_t>(c.at("max_results_per_objective"));
    (void)seed, (void)supercell, (void)radii, (void)weights, (void)iterations, (void)chunk, (void)threads;
    (void)keep, (void)mrpo;
  }
  void interact(const json& r) {
    auto objective = r.at("objective").get<T>();
    auto species = r.at("species").get<std::vector<uint8_t>>();
    auto shape = r.at("sro").at("shape").get<std::array<int, 3>>();
    auto data = r.at("sro").at("data").get<std::vector<T>>();
    if (static_cast<size_t>(shape[0]) * shape[1] * shape[2] != data.size()) throw std::runtime_error("sro shape");
    sro_values += data.size();
    (void)objective, (void)species;
  }
  void pack(const json& j) {
    const json& st = j.at("statistics");
    auto best = st.at("best_objective").get<T>();
    auto rank = st.at("best_rank").get<uint64_t>();
    auto finished = st.at("finished").get<uint64_t>();
    auto working = st.at("working").get<uint64_t>();
    for (const json& kv : st.at("timings")) {  // std::map<Timing, nanoseconds>: [name, value] pairs
      need_enum(kv.at(0), {"total", "chunk_setup", "loop", "comm", "undefined"});
      kv.at(1).get<int64_t>();
    }
    config(j.at("config"));
    const bool split = j.at("config").at("sublattice_mode").get<std::string>() == "split";
    for (const json& r : j.at("results")) {
      if (split) {
        r.at("objective").get<T>();
        for (const json& sl : r.at("sublattices")) interact(sl);
      } else {
        interact(r);
      }
      ++results;
    }
    (void)best, (void)rank, (void)finished, (void)working;
  }
};

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  std::ifstream f(argv[1], std::ios::binary);
  std::vector<uint8_t> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  try {
    const json j = json::from_msgpack(bytes);
    if (std::string(argv[2]) == "double") {
      Reader<double> r;
      r.pack(j);
      std::cout << "results " << r.results << " sro " << r.sro_values << "\n";
    } else {
      Reader<float> r;
      r.pack(j);
      std::cout << "results " << r.results << " sro " << r.sro_values << "\n";
    }
  } catch (const std::exception& e) {
    std::cerr << e.what() << "\n";
    return 1;
  }
  return 0;
}
