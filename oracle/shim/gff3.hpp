// Test infrastructure only: a minimal GFF3 reader standing in for the
// unvendored `gffsub` library (third_party/gffsub is an empty submodule in the
// reference tree). It exposes just the names src/annot.cpp uses:
// parse_file, parse_attributes, GffRecord{seqid,type,start,end,strand,
// attr_raw,id,gene_id}. Rules: tab-separated 9 columns, '#' lines skipped,
// attributes are `key=value` pairs split on ';', multi-values split on ','.
// The product's own GFF3 gene loader (eqtl_b200/host/gff.cpp) follows the
// same rules, so both sides of a parity run read a GFF identically.
#pragma once
#include <cstdint>
#include <fstream>
#include <optional>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

namespace gffsub {

enum class InputFormat { GFF3, GTF };

struct GffRecord {
  std::string seqid, source, type;
  int64_t start = 0, end = 0;
  char strand = '.';
  std::string attr_raw;
  std::optional<std::string> id, gene_id;
};

using GffData = std::vector<GffRecord>;
struct IdIndex {};

inline std::string shim_trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && (s[a] == ' ' || s[a] == '\t' || s[a] == '\r' || s[a] == '\n')) ++a;
  while (b > a && (s[b - 1] == ' ' || s[b - 1] == '\t' || s[b - 1] == '\r' || s[b - 1] == '\n')) --b;
  return s.substr(a, b - a);
}

inline std::unordered_map<std::string, std::vector<std::string>> parse_attributes(const std::string& raw) {
  std::unordered_map<std::string, std::vector<std::string>> out;
  size_t pos = 0;
  while (pos <= raw.size()) {
    size_t semi = raw.find(';', pos);
    if (semi == std::string::npos) semi = raw.size();
    std::string kv = shim_trim(raw.substr(pos, semi - pos));
    pos = semi + 1;
    if (kv.empty()) continue;
    size_t eq = kv.find('=');
    if (eq == std::string::npos) continue;
    std::string key = shim_trim(kv.substr(0, eq));
    std::string val = kv.substr(eq + 1);
    auto& vec = out[key];
    size_t vp = 0;
    while (vp <= val.size()) {
      size_t comma = val.find(',', vp);
      if (comma == std::string::npos) comma = val.size();
      vec.push_back(shim_trim(val.substr(vp, comma - vp)));
      vp = comma + 1;
    }
  }
  return out;
}

inline int parse_file(const std::string& path, GffData& data, IdIndex&, InputFormat) {
  std::ifstream in(path);
  if (!in) return 1;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::vector<std::string> col;
    size_t p = 0;
    while (true) {
      size_t t = line.find('\t', p);
      if (t == std::string::npos) { col.push_back(line.substr(p)); break; }
      col.push_back(line.substr(p, t - p));
      p = t + 1;
    }
    if (col.size() < 9) continue;
    GffRecord r;
    r.seqid = col[0];
    r.source = col[1];
    r.type = col[2];
    r.start = std::stoll(col[3]);
    r.end = std::stoll(col[4]);
    r.strand = col[6].empty() ? '.' : col[6][0];
    r.attr_raw = shim_trim(col[8]);
    auto a = parse_attributes(r.attr_raw);
    auto it = a.find("ID");
    if (it != a.end() && !it->second.empty()) r.id = it->second.front();
    it = a.find("gene_id");
    if (it != a.end() && !it->second.empty()) r.gene_id = it->second.front();
    data.push_back(std::move(r));
  }
  return 0;
}

}  // namespace gffsub
