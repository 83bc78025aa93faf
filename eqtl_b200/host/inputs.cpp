// Input files of the reference program, read with the same rules:
//   PLINK .fam/.bim/.bed        (src/plink_bed.cpp:21-120: IID = .fam column 2,
//                                SNP-major .bed with the 0x6c 0x1b 0x01 magic)
//   phenotype matrix            (src/pheno.cpp:17-88: header = sample + genes,
//                                NA / NaN / . missing, first of duplicate ids)
//   covariates                  (src/pheno.cpp:89-196: optional header row,
//                                intercept added unless a column is all 1)
//   GFF3 genes                  (src/annot.cpp:26-71: type "gene", id from
//                                --gff-id-key or ID / Name / gene_id, "gene:"
//                                prefix dropped, duplicated ids dropped,
//                                TSS = end on the minus strand)
//   GCTA GRM files              (src/grm.cpp:10-108: .grm.id IID, float32
//                                lower triangle incl. diagonal, row-major)
#include <algorithm>
#include <cerrno>
#include <cstring>
#include <fstream>
#include <sstream>
#include <unordered_set>

#include "host.hpp"

namespace eqtl_host {

namespace {

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
  while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
  return s.substr(a, b - a);
}

std::vector<std::string> split_ws(const std::string& s) {
  std::vector<std::string> out;
  std::istringstream is(s);
  std::string t;
  while (is >> t) out.push_back(t);
  return out;
}

// Tab-separated when the line has a tab, else whitespace-separated.
std::vector<std::string> split_line(const std::string& s) {
  if (s.find('\t') == std::string::npos) return split_ws(s);
  std::vector<std::string> out;
  size_t i = 0;
  while (true) {
    const size_t j = s.find('\t', i);
    out.push_back(trim(s.substr(i, j == std::string::npos ? std::string::npos : j - i)));
    if (j == std::string::npos) break;
    i = j + 1;
  }
  return out;
}

double to_double(const std::string& t, const std::string& what) {
  errno = 0;
  char* end = nullptr;
  const double v = std::strtod(t.c_str(), &end);
  if (end == t.c_str()) die("not a number in " + what + ": '" + t + "'");
  return v;
}

bool is_number(const std::string& t) {
  char* end = nullptr;
  std::strtod(t.c_str(), &end);
  return end != t.c_str();
}

}  // namespace

// ---------------------------------------------------------------- PLINK
Plink read_plink(const std::string& prefix) {
  Plink P;
  {
    std::ifstream f(prefix + ".fam");
    if (!f) die("cannot open " + prefix + ".fam");
    std::string line;
    while (std::getline(f, line)) {
      const auto t = split_ws(line);
      if (t.size() < 2) continue;
      P.fam_iid.push_back(t[1]);
    }
  }
  {
    std::ifstream f(prefix + ".bim");
    if (!f) die("cannot open " + prefix + ".bim");
    std::string line;
    while (std::getline(f, line)) {
      const auto t = split_ws(line);
      if (t.empty()) continue;
      if (t.size() < 6) die("bad .bim line: " + line);
      P.chrom.push_back(t[0]);
      P.id.push_back(t[1]);
      P.pos.push_back(std::stoll(t[3]));
      P.a1.push_back(t[4]);
      P.a2.push_back(t[5]);
    }
  }
  P.n_file = static_cast<int>(P.fam_iid.size());
  if (P.n_file == 0) die("empty .fam: " + prefix + ".fam");
  P.bytes_per_snp = (P.n_file + 3) / 4;
  const int64_t m = static_cast<int64_t>(P.chrom.size());
  FILE* fp = std::fopen((prefix + ".bed").c_str(), "rb");
  if (!fp) die("cannot open " + prefix + ".bed");
  unsigned char magic[3] = {0, 0, 0};
  if (std::fread(magic, 1, 3, fp) != 3 || magic[0] != 0x6c || magic[1] != 0x1b || magic[2] != 0x01) {
    std::fclose(fp);
    die(prefix + ".bed is not a SNP-major PLINK .bed");
  }
  P.rows.resize(static_cast<size_t>(m * P.bytes_per_snp));
  const size_t got = P.rows.empty() ? 0 : std::fread(P.rows.data(), 1, P.rows.size(), fp);
  std::fclose(fp);
  if (got != P.rows.size()) die(prefix + ".bed is shorter than .bim x .fam implies");
  return P;
}

// ----------------------------------------------------------- phenotypes
Pheno load_pheno(const std::string& path) {
  std::ifstream in(path);
  if (!in) die("cannot open pheno: " + path);
  std::string line;
  if (!std::getline(in, line)) die("empty pheno: " + path);
  line = trim(line);
  if (!line.empty() && line[0] == '#') line = line.substr(1);
  const auto header = split_line(line);
  if (header.size() < 2) die("pheno header needs sample + >=1 gene");
  Pheno P;
  for (size_t i = 1; i < header.size(); ++i) P.genes.push_back(trim(header[i]));
  {
    std::unordered_set<std::string> seen;
    for (const auto& g : P.genes)
      if (!seen.insert(g).second) die("pheno genes: duplicate id " + g);
  }
  const size_t G = P.genes.size();
  std::unordered_map<std::string, size_t> first;
  std::vector<double> row(G);
  while (std::getline(in, line)) {
    line = trim(line);
    if (line.empty() || line[0] == '#') continue;
    const auto tok = split_line(line);
    if (tok.size() != header.size())
      die("pheno row column mismatch for sample " + (tok.empty() ? std::string("?") : tok[0]));
    for (size_t j = 0; j < G; ++j) {
      const std::string& v = tok[j + 1];
      row[j] = (v == "NA" || v == "NaN" || v == ".") ? NAN : to_double(v, "pheno");
    }
    const std::string id = trim(tok[0]);
    auto it = first.find(id);
    if (it != first.end()) {
      const double* prev = &P.Y[it->second * G];
      for (size_t j = 0; j < G; ++j)
        if (!(std::isnan(prev[j]) && std::isnan(row[j])) && !(prev[j] == row[j]))
          die("pheno samples: duplicate id with conflicting values: " + id);
      continue;
    }
    first.emplace(id, P.samples.size());
    P.samples.push_back(id);
    P.Y.insert(P.Y.end(), row.begin(), row.end());
  }
  if (P.samples.empty()) die("no samples in pheno");
  return P;
}

// ----------------------------------------------------------- covariates
std::vector<double> load_covar(const std::string& path, const std::vector<std::string>& samples, int& p) {
  const size_t n = samples.size();
  if (path.empty()) {
    p = 1;
    return std::vector<double>(n, 1.0);
  }
  std::ifstream in(path);
  if (!in) die("cannot open covar: " + path);
  std::vector<std::string> ids;
  std::vector<std::vector<double>> rows;
  std::string line;
  bool first = true;
  while (std::getline(in, line)) {
    line = trim(line);
    if (line.empty() || line[0] == '#') continue;
    const auto t = split_line(line);
    if (t.size() < 2) continue;
    if (first) {
      first = false;
      if (!is_number(t[1])) continue;  // header row
    }
    std::vector<double> r;
    for (size_t j = 1; j < t.size(); ++j) r.push_back(to_double(t[j], "covar"));
    ids.push_back(t[0]);
    rows.push_back(std::move(r));
  }
  if (rows.empty()) die("no covariates in " + path);
  const size_t nc = rows[0].size();
  std::unordered_map<std::string, size_t> at;
  for (size_t i = 0; i < ids.size(); ++i) {
    auto it = at.find(ids[i]);
    if (it == at.end()) {
      at.emplace(ids[i], i);
    } else if (rows[it->second] != rows[i]) {
      die("covar samples: duplicate id with conflicting values: " + ids[i]);
    }
  }
  std::vector<double> raw(n * nc);
  for (size_t i = 0; i < n; ++i) {
    auto it = at.find(samples[i]);
    if (it == at.end()) die("sample " + samples[i] + " missing in covar");
    if (rows[it->second].size() != nc) die("covar row width mismatch");
    for (size_t j = 0; j < nc; ++j) raw[j * n + i] = rows[it->second][j];
  }
  bool has_int = false;
  for (size_t j = 0; j < nc && !has_int; ++j) {
    bool ok = true;
    for (size_t i = 0; i < n && ok; ++i) ok = std::fabs(raw[j * n + i] - 1.0) <= 1e-12;
    has_int = ok;
  }
  if (has_int) {
    p = static_cast<int>(nc);
    return raw;
  }
  std::vector<double> X(n * (nc + 1), 1.0);
  std::copy(raw.begin(), raw.end(), X.begin() + n);
  p = static_cast<int>(nc + 1);
  return X;
}

// ------------------------------------------------------------------ GFF
std::unordered_map<std::string, GeneLoc> load_gff(const std::string& path, const std::string& id_key) {
  std::ifstream in(path);
  if (!in) die("cannot open gff: " + path);
  std::unordered_map<std::string, GeneLoc> out;
  std::unordered_set<std::string> multi;
  std::string line;
  while (std::getline(in, line)) {
    if (line.empty() || line[0] == '#') continue;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::vector<std::string> c;
    size_t i = 0;
    while (true) {
      const size_t j = line.find('\t', i);
      c.push_back(line.substr(i, j == std::string::npos ? std::string::npos : j - i));
      if (j == std::string::npos) break;
      i = j + 1;
    }
    if (c.size() < 9 || c[2] != "gene") continue;
    std::unordered_map<std::string, std::string> attrs;
    const std::string a = trim(c[8]);
    size_t k = 0;
    while (k <= a.size()) {
      size_t e = a.find(';', k);
      if (e == std::string::npos) e = a.size();
      const std::string kv = trim(a.substr(k, e - k));
      const size_t eq = kv.find('=');
      if (eq != std::string::npos) {
        const std::string key = trim(kv.substr(0, eq));
        std::string val = kv.substr(eq + 1);
        val = trim(val.substr(0, val.find(',')));
        attrs.emplace(key, val);
      }
      k = e + 1;
    }
    auto get = [&](const char* key) {
      auto it = attrs.find(key);
      return it == attrs.end() ? std::string() : it->second;
    };
    std::string gid;
    if (!id_key.empty()) {
      gid = get(id_key.c_str());
    } else {
      gid = get("ID");
      if (gid.empty()) gid = get("Name");
      if (gid.empty()) gid = get("gene_id");
    }
    if (gid.empty()) continue;
    if (gid.rfind("gene:", 0) == 0) gid = gid.substr(5);
    if (multi.count(gid)) continue;
    if (out.count(gid)) {
      out.erase(gid);
      multi.insert(gid);
      continue;
    }
    GeneLoc L;
    L.chrom = c[0];
    L.start = std::stoll(c[3]);
    L.end = std::stoll(c[4]);
    L.tss = c[6] == "-" ? L.end : L.start;
    out.emplace(gid, L);
  }
  return out;
}

std::string chrom_key(const std::string& c) {
  std::string s = c;
  if (s.size() >= 3 && (s[0] == 'c' || s[0] == 'C') && (s[1] == 'h' || s[1] == 'H') && (s[2] == 'r' || s[2] == 'R'))
    s = s.substr(3);
  size_t i = 0;
  while (i + 1 < s.size() && s[i] == '0') ++i;
  return s.substr(i);
}

// ------------------------------------------------------------------ GRM
GrmFile load_grm(const std::string& prefix) {
  GrmFile g;
  std::ifstream idf(prefix + ".grm.id");
  if (!idf) die("cannot open " + prefix + ".grm.id");
  std::string line;
  while (std::getline(idf, line)) {
    const auto t = split_ws(line);
    if (t.size() >= 2) g.ids.push_back(t[1]);
    else if (t.size() == 1) g.ids.push_back(t[0]);
  }
  const size_t n = g.ids.size();
  if (n == 0) die("empty GRM id file");
  const size_t ntri = n * (n + 1) / 2;
  std::vector<float> buf(ntri);
  FILE* fp = std::fopen((prefix + ".grm.bin").c_str(), "rb");
  if (!fp) die("cannot open " + prefix + ".grm.bin");
  const size_t got = std::fread(buf.data(), sizeof(float), ntri, fp);
  std::fclose(fp);
  if (got != ntri) die("GRM bin size mismatch");
  g.K.assign(n * n, 0.0);
  size_t k = 0;
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j <= i; ++j) {
      const double v = buf[k++];
      g.K[i * n + j] = v;
      g.K[j * n + i] = v;
    }
  return g;
}

std::vector<double> slice_grm(const GrmFile& g, const std::vector<std::string>& samples) {
  std::unordered_map<std::string, size_t> at;
  for (size_t i = 0; i < g.ids.size(); ++i) at.emplace(g.ids[i], i);
  const size_t n = samples.size(), N = g.ids.size();
  std::vector<size_t> ix(n);
  for (size_t i = 0; i < n; ++i) {
    auto it = at.find(samples[i]);
    if (it == at.end()) die("sample missing in GRM: " + samples[i]);
    ix[i] = it->second;
  }
  std::vector<double> K(n * n);
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j < n; ++j) K[i * n + j] = g.K[ix[i] * N + ix[j]];
  return K;
}

void write_grm(const std::string& prefix, const std::vector<std::string>& ids, const std::vector<double>& K,
               const std::vector<int32_t>& N_packed) {
  const size_t n = ids.size();
  {
    std::ofstream idf(prefix + ".grm.id");
    if (!idf) die("cannot write " + prefix + ".grm.id");
    for (const auto& id : ids) idf << id << '\t' << id << '\n';
  }
  const size_t ntri = n * (n + 1) / 2;
  std::vector<float> buf(ntri);
  size_t k = 0;
  for (size_t i = 0; i < n; ++i)
    for (size_t j = 0; j <= i; ++j) buf[k++] = static_cast<float>(K[i * n + j]);
  auto dump = [&](const std::string& path) {
    FILE* fp = std::fopen(path.c_str(), "wb");
    if (!fp) die("cannot write " + path);
    std::fwrite(buf.data(), sizeof(float), ntri, fp);
    std::fclose(fp);
  };
  dump(prefix + ".grm.bin");
  if (!N_packed.empty()) {
    if (N_packed.size() != ntri) die("GRM N_packed size mismatch on write");
    for (size_t i = 0; i < ntri; ++i) buf[i] = static_cast<float>(N_packed[i]);
    dump(prefix + ".grm.N.bin");
  }
}

}  // namespace eqtl_host
