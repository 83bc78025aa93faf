// VCF input: the GT calls of a plain or bgzip/gzip-compressed VCF, read the
// way the reference's VcfSession reads them (src/vcf_session.cpp:160-305),
// into the same 2-bit SNP-major rows as a PLINK .bed so that the device path
// is shared: ALT is the counted allele (A1), REF the other (A2); code 00 = 2
// ALT alleles, 10 = 1, 11 = 0, 01 = missing. Only biallelic records are kept
// (multi-allelic ones are counted and skipped); BCF is refused.
//
// The reference filters VCF records with a ploidy-aware allele frequency:
// on X, Y and MT (and for any haploid call) a call carries one allele, so
// af = sum of ALT counts / sum of ploidies, not mean / 2. vcf_filter applies
// those filters on the host over the analysis samples; the device then sees
// only records that pass and applies no filter of its own (its mean / 2
// frequency would disagree there). Imputation (mean of the non-missing
// calls), the GRM and the per-gene subset gate use the dosages alone and are
// the same for both inputs.
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>

#include "host.hpp"

namespace eqtl_host {

namespace {

// A header that defines the ID "DS" (INFO, FORMAT or FILTER) switches the
// reader to dosage rows (src/vcf_session.cpp:66-68): a record whose FORMAT
// carries DS, declared Type=Float, gives each sample's first DS value as its
// dosage (".", an absent subfield or a value that is not a finite number is
// missing; the value is used as it is, as an FP32 number); any other record
// gives its GT counts (:193-258). Both kinds then share the FP32 rows.
//
// Line reader over gzread (which also reads uncompressed files as they are).
struct GzLines {
  gzFile f = nullptr;
  std::vector<char> buf;
  size_t beg = 0, end = 0;
  bool eof = false;
  explicit GzLines(const std::string& path) : buf(1 << 20) {
    f = gzopen(path.c_str(), "rb");
    if (!f) die("cannot open VCF/BCF: " + path);
    gzbuffer(f, 1 << 18);
  }
  ~GzLines() {
    if (f) gzclose(f);
  }
  // next line without its newline; false at the end of the file
  bool next(std::string& line) {
    line.clear();
    while (true) {
      const char* s = buf.data() + beg;
      const void* nl = beg < end ? std::memchr(s, '\n', end - beg) : nullptr;
      if (nl) {
        const size_t len = static_cast<const char*>(nl) - s;
        line.append(s, len);
        beg += len + 1;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        return true;
      }
      line.append(s, end - beg);
      beg = end = 0;
      if (eof) return !line.empty();
      const int got = gzread(f, buf.data(), static_cast<unsigned>(buf.size()));
      if (got < 0) die("VCF read error");
      if (got == 0) eof = true;
      end = static_cast<size_t>(got);
    }
  }
};

// X, Y and MT, with or without a "chr" prefix (src/vcf_session.cpp:148-157)
bool haploid_chrom(const std::string& chrom) {
  std::string k = chrom;
  if (k.size() > 3 && (k[0] == 'c' || k[0] == 'C') && (k[1] == 'h' || k[1] == 'H') && (k[2] == 'r' || k[2] == 'R'))
    k = k.substr(3);
  return k == "X" || k == "x" || k == "Y" || k == "y" || k == "M" || k == "m" || k == "MT" || k == "mt" ||
         k == "Mt";
}

// One GT value: ALT dosage, or -1 if missing; `haploid` when one allele is
// present. The first two alleles count (bcf_get_genotypes' first two slots).
int parse_gt(const char* s, size_t len, bool& haploid) {
  int alleles[2] = {-2, -2};  // -2 absent, -1 missing
  int na = 0;
  size_t i = 0;
  while (i < len && na < 2) {
    if (s[i] == '.') {
      alleles[na++] = -1;
      ++i;
    } else if (s[i] >= '0' && s[i] <= '9') {
      int v = 0;
      while (i < len && s[i] >= '0' && s[i] <= '9') v = 10 * v + (s[i++] - '0');
      alleles[na++] = v;
    } else {
      die("malformed GT value in VCF: " + std::string(s, len));
    }
    if (i < len && (s[i] == '/' || s[i] == '|')) ++i;
    else break;
  }
  if (na == 0 || alleles[0] == -1 || alleles[1] == -1) return -1;  // ".", "./.", "0/."
  int d = alleles[0];
  haploid = alleles[1] == -2;
  if (!haploid) d += alleles[1];
  if (alleles[0] > 1 || alleles[1] > 1) die("VCF GT allele index beyond the single ALT allele");
  return d;
}

// [begin, end) of the k-th ':'-separated subfield of a sample column, or
// false when the column has fewer subfields.
bool subfield(const char* s, size_t len, int k, size_t& p0, size_t& p1) {
  p0 = 0;
  for (int j = 0; j < k; ++j) {
    const void* c = p0 < len ? std::memchr(s + p0, ':', len - p0) : nullptr;
    if (!c) return false;
    p0 = static_cast<const char*>(c) - s + 1;
  }
  p1 = p0;
  while (p1 < len && s[p1] != ':') ++p1;
  return true;
}

// The ID of a ##INFO / ##FORMAT / ##FILTER header line, and its Type.
void header_id(const std::string& line, std::string& id, std::string& type) {
  id.clear();
  type.clear();
  const size_t lt = line.find('<');
  if (lt == std::string::npos) return;
  // the key=value pairs before any quoted text (Description="...")
  const std::string body = line.substr(lt + 1, line.find('"') == std::string::npos ? std::string::npos
                                                                                     : line.find('"') - lt - 1);
  size_t a = 0;
  while (a < body.size()) {
    size_t e = body.find_first_of(",>", a);
    if (e == std::string::npos) e = body.size();
    const std::string kv = body.substr(a, e - a);
    if (kv.compare(0, 3, "ID=") == 0) id = kv.substr(3);
    if (kv.compare(0, 5, "Type=") == 0) type = kv.substr(5);
    a = e + 1;
  }
}

// One DS value: the first number of the subfield, NaN when missing.
float parse_ds(const char* s, size_t len) {
  if (len == 0 || (len == 1 && s[0] == '.')) return std::numeric_limits<float>::quiet_NaN();
  std::string t(s, len);
  const size_t comma = t.find(',');
  if (comma != std::string::npos) t.resize(comma);
  char* end = nullptr;
  const double v = std::strtod(t.c_str(), &end);
  if (end == t.c_str()) return std::numeric_limits<float>::quiet_NaN();
  const float f = static_cast<float>(v);
  return std::isfinite(f) ? f : std::numeric_limits<float>::quiet_NaN();
}

}  // namespace

Plink read_vcf(const std::string& path, VcfInfo& vi) {
  GzLines in(path);
  Plink P;
  std::string line;
  bool have_header = false;
  if (!in.next(line)) die("empty VCF: " + path);
  if (line.compare(0, 3, "BCF") == 0)
    die("BCF input is not read by this build; convert with bcftools view -Oz to a VCF");
  std::vector<const char*> fld;
  std::vector<size_t> flen;
  int64_t n_rec = 0;
  bool prefer_ds = false, ds_float = false, said_ds = false;
  do {
    if (line.empty()) continue;
    if (line[0] == '#') {
      const bool fmt_line = line.compare(0, 10, "##FORMAT=<") == 0;
      if (fmt_line || line.compare(0, 8, "##INFO=<") == 0 || line.compare(0, 10, "##FILTER=<") == 0) {
        std::string id, type;
        header_id(line, id, type);
        if (id == "DS") {
          prefer_ds = true;
          if (fmt_line) ds_float = type == "Float";
        }
      }
      if (line.compare(0, 6, "#CHROM") == 0) {
        size_t a = 0;
        int col = 0;
        while (a <= line.size()) {
          size_t b = line.find('\t', a);
          if (b == std::string::npos) b = line.size();
          if (col >= 9) P.fam_iid.push_back(line.substr(a, b - a));
          ++col;
          a = b + 1;
        }
        have_header = true;
        P.n_file = static_cast<int>(P.fam_iid.size());
        P.bytes_per_snp = (P.n_file + 3) / 4;
        if (P.n_file == 0) die("VCF has no samples: " + path);
        P.dense = prefer_ds;
        if (prefer_ds) info("VCF: FORMAT/DS present -> use dosage field when available");
      }
      continue;
    }
    if (!have_header) die("VCF record before the #CHROM header line: " + path);
    ++n_rec;
    fld.clear();
    flen.clear();
    size_t a = 0;
    while (a <= line.size()) {
      size_t b = line.find('\t', a);
      if (b == std::string::npos) b = line.size();
      fld.push_back(line.data() + a);
      flen.push_back(b - a);
      a = b + 1;
    }
    if (fld.size() < 9 + static_cast<size_t>(P.n_file)) die("VCF record with fewer sample columns than the header");
    const std::string alt(fld[4], flen[4]);
    if (alt == "." || alt.find(',') != std::string::npos) {  // not biallelic (n_allele != 2)
      ++vi.n_multi;
      continue;
    }
    // GT's and DS's positions among the FORMAT keys
    int gt_at = -1, ds_at = -1;
    {
      int k = 0;
      size_t s = 0;
      const std::string fmt(fld[8], flen[8]);
      while (s <= fmt.size()) {
        size_t e = fmt.find(':', s);
        if (e == std::string::npos) e = fmt.size();
        if (fmt.compare(s, e - s, "GT") == 0) gt_at = k;
        if (fmt.compare(s, e - s, "DS") == 0) ds_at = k;
        ++k;
        s = e + 1;
      }
    }
    const bool use_ds = prefer_ds && ds_float && ds_at >= 0;
    if (!use_ds && gt_at < 0) continue;  // no genotypes in this record
    if (use_ds && !said_ds) {
      info("VCF: using FORMAT/DS dosages");
      said_ds = true;
    }
    const std::string chrom(fld[0], flen[0]);
    const bool hap = haploid_chrom(chrom);
    std::vector<uint8_t> row(P.dense ? 0 : static_cast<size_t>(P.bytes_per_snp), 0);
    std::vector<float> drow(P.dense ? static_cast<size_t>(P.n_file) : 0);
    std::vector<int32_t> hap_calls;
    for (int i = 0; i < P.n_file; ++i) {
      const char* s = fld[9 + i];
      const size_t len = flen[9 + i];
      size_t p0 = 0, p1 = 0;
      if (use_ds) {
        drow[static_cast<size_t>(i)] = subfield(s, len, ds_at, p0, p1) ? parse_ds(s + p0, p1 - p0)
                                                                         : std::numeric_limits<float>::quiet_NaN();
        continue;
      }
      // the GT subfield of this sample (absent trailing subfields are missing)
      bool haploid = false;
      const int d = (subfield(s, len, gt_at, p0, p1) && p1 > p0) ? parse_gt(s + p0, p1 - p0, haploid) : -1;
      if (P.dense) {
        drow[static_cast<size_t>(i)] = d < 0 ? std::numeric_limits<float>::quiet_NaN() : static_cast<float>(d);
      } else {
        const uint32_t code = d < 0 ? 1u : (d == 2 ? 0u : (d == 1 ? 2u : 3u));
        row[static_cast<size_t>(i >> 2)] |= static_cast<uint8_t>(code << ((i & 3) * 2));
      }
      if (d >= 0 && haploid && !hap) hap_calls.push_back(i);
    }
    P.chrom.push_back(chrom);
    P.pos.push_back(std::stoll(std::string(fld[1], flen[1])));
    const std::string id(fld[2], flen[2]);
    P.id.push_back(id == "." ? std::string() : id);
    P.a2.push_back(std::string(fld[3], flen[3]));  // REF
    P.a1.push_back(alt);                            // ALT, the counted allele
    P.rows.insert(P.rows.end(), row.begin(), row.end());
    P.ds.insert(P.ds.end(), drow.begin(), drow.end());
    vi.hap_chrom.push_back(hap ? 1 : 0);
    vi.hap_calls.push_back(std::move(hap_calls));
  } while (in.next(line));
  if (!have_header) die("VCF without a #CHROM header line: " + path);
  if (vi.n_multi > 0)
    info("VCF multi-allelic sites skipped (biallelic only): " + std::to_string(vi.n_multi));
  info("VCF: " + std::to_string(P.chrom.size()) + " biallelic records of " + std::to_string(n_rec) + " on " +
       std::to_string(P.n_file) + " samples");
  return P;
}

bool vcf_has_index(const std::string& path) {
  for (const char* ext : {".tbi", ".csi"}) {
    gzFile f = gzopen((path + ext).c_str(), "rb");
    if (!f) continue;
    char magic[4] = {0, 0, 0, 0};
    const int got = gzread(f, magic, 4);
    gzclose(f);
    if (got == 4 && magic[3] == 1 &&
        ((magic[0] == 'T' && magic[1] == 'B' && magic[2] == 'I') || (magic[0] == 'C' && magic[1] == 'S' && magic[2] == 'I')))
      return true;
  }
  return false;
}

void vcf_filter(Plink& P, const VcfInfo& vi, const std::vector<int32_t>& cols, const Options& opt) {
  const int64_t m = static_cast<int64_t>(P.chrom.size());
  const int n_an = static_cast<int>(cols.size());
  std::vector<uint8_t> keep(static_cast<size_t>(m), 0);
  for (int64_t s = 0; s < m; ++s) {
    const std::vector<int32_t>& hc = vi.hap_calls[static_cast<size_t>(s)];
    int n_miss = 0, n_ok = 0;
    double sum = 0.0, ploidy = 0.0;
    for (int i = 0; i < n_an; ++i) {
      const int c = cols[i];
      double d;
      if (P.dense) {
        d = static_cast<double>(P.ds[static_cast<size_t>(s) * P.n_file + c]);
      } else {
        const uint32_t code = (P.rows[s * P.bytes_per_snp + (c >> 2)] >> ((c & 3) * 2)) & 3u;
        d = code == 1u ? std::numeric_limits<double>::quiet_NaN() : (code == 0u ? 2.0 : (code == 2u ? 1.0 : 0.0));
      }
      if (std::isnan(d)) {
        ++n_miss;
        continue;
      }
      sum += d;
      const bool hap = vi.hap_chrom[static_cast<size_t>(s)] || std::binary_search(hc.begin(), hc.end(), c);
      ploidy += hap ? 1.0 : 2.0;
      ++n_ok;
    }
    if (n_ok == 0) continue;
    if (static_cast<double>(n_miss) / static_cast<double>(n_an) > opt.max_miss + 1e-15) continue;
    double af = ploidy > 0 ? sum / ploidy : 0.0;
    af = std::min(std::max(af, 0.0), 1.0);
    if (af < 1e-12 || af > 1.0 - 1e-12) continue;  // monomorphic
    if (opt.miss_filter && n_miss > 0) continue;
    if (opt.maf > 0.0 && (af < opt.maf || af > 1.0 - opt.maf)) continue;  // pass_maf
    keep[static_cast<size_t>(s)] = 1;
  }
  int64_t n_pass = 0;
  for (uint8_t k : keep) n_pass += k;
  info("VCF: " + std::to_string(n_pass) + " of " + std::to_string(m) + " biallelic records pass the filters on " +
       std::to_string(n_an) + " samples");
  // compact to the records that pass
  Plink Q;
  Q.fam_iid = P.fam_iid;
  Q.n_file = P.n_file;
  Q.bytes_per_snp = P.bytes_per_snp;
  Q.dense = P.dense;
  for (int64_t s = 0; s < m; ++s) {
    if (!keep[static_cast<size_t>(s)]) continue;
    Q.chrom.push_back(P.chrom[s]);
    Q.pos.push_back(P.pos[s]);
    Q.id.push_back(P.id[s]);
    Q.a1.push_back(P.a1[s]);
    Q.a2.push_back(P.a2[s]);
    if (P.dense)
      Q.ds.insert(Q.ds.end(), P.ds.begin() + s * P.n_file, P.ds.begin() + (s + 1) * P.n_file);
    else
      Q.rows.insert(Q.rows.end(), P.rows.begin() + s * P.bytes_per_snp, P.rows.begin() + (s + 1) * P.bytes_per_snp);
  }
  P = std::move(Q);
}

}  // namespace eqtl_host
