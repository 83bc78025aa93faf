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
#include <cstring>

#include "host.hpp"

namespace eqtl_host {

namespace {

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
  do {
    if (line.empty()) continue;
    if (line[0] == '#') {
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
    // GT's position among the FORMAT keys
    int gt_at = -1;
    {
      int k = 0;
      size_t s = 0;
      const std::string fmt(fld[8], flen[8]);
      while (s <= fmt.size()) {
        size_t e = fmt.find(':', s);
        if (e == std::string::npos) e = fmt.size();
        if (fmt.compare(s, e - s, "GT") == 0) gt_at = k;
        ++k;
        s = e + 1;
      }
    }
    if (gt_at < 0) continue;  // no genotypes in this record
    const std::string chrom(fld[0], flen[0]);
    const bool hap = haploid_chrom(chrom);
    std::vector<uint8_t> row(static_cast<size_t>(P.bytes_per_snp), 0);
    std::vector<int32_t> hap_calls;
    for (int i = 0; i < P.n_file; ++i) {
      const char* s = fld[9 + i];
      const size_t len = flen[9 + i];
      // the GT subfield of this sample (absent trailing subfields are missing)
      size_t p0 = 0;
      int k = 0;
      while (k < gt_at && p0 < len) {
        const void* c = std::memchr(s + p0, ':', len - p0);
        if (!c) {
          p0 = len;
          break;
        }
        p0 = static_cast<const char*>(c) - s + 1;
        ++k;
      }
      size_t p1 = p0;
      while (p1 < len && s[p1] != ':') ++p1;
      bool haploid = false;
      const int d = (k == gt_at && p1 > p0) ? parse_gt(s + p0, p1 - p0, haploid) : -1;
      const uint32_t code = d < 0 ? 1u : (d == 2 ? 0u : (d == 1 ? 2u : 3u));
      row[static_cast<size_t>(i >> 2)] |= static_cast<uint8_t>(code << ((i & 3) * 2));
      if (d >= 0 && haploid && !hap) hap_calls.push_back(i);
    }
    P.chrom.push_back(chrom);
    P.pos.push_back(std::stoll(std::string(fld[1], flen[1])));
    const std::string id(fld[2], flen[2]);
    P.id.push_back(id == "." ? std::string() : id);
    P.a2.push_back(std::string(fld[3], flen[3]));  // REF
    P.a1.push_back(alt);                            // ALT, the counted allele
    P.rows.insert(P.rows.end(), row.begin(), row.end());
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

void vcf_filter(Plink& P, const VcfInfo& vi, const std::vector<int32_t>& cols, const Options& opt) {
  const int64_t m = static_cast<int64_t>(P.chrom.size());
  const int n_an = static_cast<int>(cols.size());
  std::vector<uint8_t> keep(static_cast<size_t>(m), 0);
  for (int64_t s = 0; s < m; ++s) {
    const uint8_t* row = P.rows.data() + s * P.bytes_per_snp;
    const std::vector<int32_t>& hc = vi.hap_calls[static_cast<size_t>(s)];
    int n_miss = 0, n_ok = 0;
    double sum = 0.0, ploidy = 0.0;
    for (int i = 0; i < n_an; ++i) {
      const int c = cols[i];
      const uint32_t code = (row[c >> 2] >> ((c & 3) * 2)) & 3u;
      if (code == 1u) {
        ++n_miss;
        continue;
      }
      sum += code == 0u ? 2.0 : (code == 2u ? 1.0 : 0.0);
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
  for (int64_t s = 0; s < m; ++s) {
    if (!keep[static_cast<size_t>(s)]) continue;
    Q.chrom.push_back(P.chrom[s]);
    Q.pos.push_back(P.pos[s]);
    Q.id.push_back(P.id[s]);
    Q.a1.push_back(P.a1[s]);
    Q.a2.push_back(P.a2[s]);
    Q.rows.insert(Q.rows.end(), P.rows.begin() + s * P.bytes_per_snp, P.rows.begin() + (s + 1) * P.bytes_per_snp);
  }
  P = std::move(Q);
}

}  // namespace eqtl_host
