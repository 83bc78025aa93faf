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
#include <atomic>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <thread>

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

namespace {

// The whole file as text: a BGZF file (gzip members with the BC extra field,
// each member at most 64 KiB of text) is inflated member by member on all
// host threads, any other gzip stream through gzread, plain text as it is.
std::string read_all(const std::string& path) {
  std::string raw;
  {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) die("cannot open VCF/BCF: " + path);
    char buf[1 << 16];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) raw.append(buf, got);
    std::fclose(f);
  }
  const auto u8 = [&](size_t k) { return static_cast<uint8_t>(raw[k]); };
  const auto le16 = [&](size_t k) { return static_cast<uint32_t>(u8(k)) | (static_cast<uint32_t>(u8(k + 1)) << 8); };
  const auto le32 = [&](size_t k) { return le16(k) | (le16(k + 2) << 16); };
  if (raw.size() < 2 || u8(0) != 0x1f || u8(1) != 0x8b) return raw;  // plain text
  // BGZF members: (offset, compressed data offset, data bytes, text bytes)
  struct Member {
    size_t off, data, len, isize;
  };
  std::vector<Member> mem;
  bool bgzf = true;
  for (size_t off = 0; off < raw.size() && bgzf;) {
    if (off + 18 > raw.size() || u8(off) != 0x1f || u8(off + 1) != 0x8b || u8(off + 2) != 8 || !(u8(off + 3) & 4)) {
      bgzf = false;
      break;
    }
    const size_t xlen = le16(off + 10);
    size_t bsize = 0;
    for (size_t x = off + 12; x + 4 <= off + 12 + xlen && x + 4 <= raw.size();) {
      const size_t slen = le16(x + 2);
      if (u8(x) == 'B' && u8(x + 1) == 'C' && slen == 2) bsize = le16(x + 4) + 1;
      x += 4 + slen;
    }
    if (bsize == 0 || off + bsize > raw.size() || bsize < 12 + xlen + 8) {
      bgzf = false;
      break;
    }
    mem.push_back({off, off + 12 + xlen, bsize - 12 - xlen - 8, le32(off + bsize - 4)});
    off += bsize;
  }
  if (!bgzf) {  // a gzip stream that is not BGZF
    gzFile f = gzopen(path.c_str(), "rb");
    if (!f) die("cannot open VCF/BCF: " + path);
    std::string text;
    std::vector<char> buf(1 << 20);
    int got;
    while ((got = gzread(f, buf.data(), static_cast<unsigned>(buf.size()))) > 0) text.append(buf.data(), got);
    const bool err = got < 0;
    gzclose(f);
    if (err) die("VCF read error");
    return text;
  }
  std::vector<size_t> at(mem.size() + 1, 0);
  for (size_t k = 0; k < mem.size(); ++k) at[k + 1] = at[k] + mem[k].isize;
  std::string text(at.back(), '\0');
  std::atomic<bool> bad{false};
  const size_t nt = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), mem.size()));
  std::vector<std::thread> th;
  for (size_t t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      for (size_t k = t; k < mem.size(); k += nt) {
        if (mem[k].isize == 0) continue;
        z_stream zs{};
        if (inflateInit2(&zs, -15) != Z_OK) {
          bad = true;
          return;
        }
        zs.next_in = reinterpret_cast<Bytef*>(&raw[mem[k].data]);
        zs.avail_in = static_cast<uInt>(mem[k].len);
        zs.next_out = reinterpret_cast<Bytef*>(&text[at[k]]);
        zs.avail_out = static_cast<uInt>(mem[k].isize);
        const int rc = inflate(&zs, Z_FINISH);
        if (rc != Z_STREAM_END || zs.total_out != mem[k].isize) bad = true;
        inflateEnd(&zs);
      }
    });
  for (auto& x : th) x.join();
  if (bad) die("VCF read error (BGZF member)");
  return text;
}

}  // namespace

namespace {

// ------------------------------------------------------------------- BCF
// BCF2 (the VCF specification's binary form, as htslib writes it): "BCF\2\x"
// magic, the header text, then records of shared fields (CHROM as a contig
// index, 0-based POS, ID, alleles, FILTER, INFO) and per-FORMAT-key sample
// arrays of typed values. Sentinels: int8/16/32 missing 0x80.., vector end
// 0x80..01; float missing 0x7F800001, vector end 0x7F800002. GT values are
// (allele + 1) << 1 | phased, 0 for a missing allele.
struct BcfReader {
  const std::string& b;
  size_t at;
  explicit BcfReader(const std::string& buf, size_t off) : b(buf), at(off) {}
  void need(size_t k) const {
    if (at + k > b.size()) die("BCF record truncated");
  }
  uint32_t u32() {
    need(4);
    uint32_t v;
    std::memcpy(&v, b.data() + at, 4);
    at += 4;
    return v;
  }
  uint8_t u8() {
    need(1);
    return static_cast<uint8_t>(b[at++]);
  }
  // typed descriptor: (type, count)
  void desc(int& type, int64_t& count) {
    const uint8_t d = u8();
    type = d & 15;
    count = d >> 4;
    if (count == 15) count = int_value();
  }
  int64_t int_value() {
    int t;
    int64_t c;
    desc(t, c);
    if (c != 1) die("BCF typed integer with count " + std::to_string(c));
    return scalar_int(t);
  }
  int64_t scalar_int(int t) {
    if (t == 1) return static_cast<int8_t>(u8());
    if (t == 2) {
      need(2);
      int16_t v;
      std::memcpy(&v, b.data() + at, 2);
      at += 2;
      return v;
    }
    if (t == 3) return static_cast<int32_t>(u32());
    die("BCF typed value of type " + std::to_string(t) + " where an integer is expected");
  }
  static size_t width(int t) { return t == 1 || t == 7 ? 1 : (t == 2 ? 2 : (t == 3 || t == 5 ? 4 : 0)); }
  std::string string_value() {
    int t;
    int64_t c;
    desc(t, c);
    if (c > 0 && t != 7) die("BCF typed string of type " + std::to_string(t));
    need(static_cast<size_t>(c));
    std::string s(b.data() + at, static_cast<size_t>(c));
    at += static_cast<size_t>(c);
    const size_t z = s.find('\0');
    if (z != std::string::npos) s.resize(z);
    return s;
  }
  void skip_typed() {
    int t;
    int64_t c;
    desc(t, c);
    const size_t w = width(t);
    if (c > 0 && w == 0) die("BCF typed value of unknown type " + std::to_string(t));
    need(w * static_cast<size_t>(c));
    at += w * static_cast<size_t>(c);
  }
};

// one element of an integer array of type t, widened with the sentinels
// mapped to int32's (missing INT32_MIN, vector end INT32_MIN + 1)
int32_t widen(const char* p, int t) {
  if (t == 1) {
    const int8_t v = static_cast<int8_t>(*p);
    return v == INT8_MIN ? INT32_MIN : (v == INT8_MIN + 1 ? INT32_MIN + 1 : v);
  }
  if (t == 2) {
    int16_t v;
    std::memcpy(&v, p, 2);
    return v == INT16_MIN ? INT32_MIN : (v == INT16_MIN + 1 ? INT32_MIN + 1 : v);
  }
  int32_t v;
  std::memcpy(&v, p, 4);
  return v;
}

Plink read_bcf_records(const std::string& text, VcfInfo& vi) {
  if (text.size() < 9 || static_cast<uint8_t>(text[3]) != 2)
    die("BCF input of an unsupported version (BCF2 is read)");
  uint32_t l_text;
  std::memcpy(&l_text, text.data() + 5, 4);
  if (9 + static_cast<size_t>(l_text) > text.size()) die("BCF header truncated");
  std::string header(text.data() + 9, l_text);
  const size_t z = header.find('\0');
  if (z != std::string::npos) header.resize(z);
  Plink P;
  // the string dictionary (PASS first) and the contig dictionary, in header
  // order unless an IDX attribute says otherwise
  std::vector<std::string> dict{"PASS"}, contigs;
  auto put = [](std::vector<std::string>& d, const std::string& id, int idx) {
    if (idx >= 0) {
      if (static_cast<size_t>(idx) >= d.size()) d.resize(static_cast<size_t>(idx) + 1);
      d[static_cast<size_t>(idx)] = id;
    } else if (std::find(d.begin(), d.end(), id) == d.end()) {
      d.push_back(id);
    }
  };
  auto attr = [](const std::string& line, const std::string& key) -> std::string {
    const size_t lt = line.find('<');
    if (lt == std::string::npos) return "";
    const std::string body = line.substr(lt + 1);
    size_t a = 0;
    while (a < body.size()) {
      if (body[a] == '"') {  // skip quoted text
        const size_t q = body.find('"', a + 1);
        a = q == std::string::npos ? body.size() : q + 1;
        continue;
      }
      const size_t e = body.find_first_of(",>", a);
      const std::string kv = body.substr(a, (e == std::string::npos ? body.size() : e) - a);
      if (kv.compare(0, key.size() + 1, key + "=") == 0) return kv.substr(key.size() + 1);
      if (e == std::string::npos) break;
      a = e + 1;
    }
    return "";
  };
  bool prefer_ds = false, ds_float = false, said_ds = false;
  size_t ls = 0;
  while (ls < header.size()) {
    size_t le = header.find('\n', ls);
    if (le == std::string::npos) le = header.size();
    std::string line = header.substr(ls, le - ls);
    if (!line.empty() && line.back() == '\r') line.pop_back();
    ls = le + 1;
    const bool fmt_line = line.compare(0, 10, "##FORMAT=<") == 0;
    if (fmt_line || line.compare(0, 8, "##INFO=<") == 0 || line.compare(0, 10, "##FILTER=<") == 0) {
      std::string id, type;
      header_id(line, id, type);
      const std::string idx = attr(line, "IDX");
      put(dict, id, idx.empty() ? -1 : std::atoi(idx.c_str()));
      if (id == "DS") {
        prefer_ds = true;
        if (fmt_line) ds_float = type == "Float";
      }
    } else if (line.compare(0, 10, "##contig=<") == 0) {
      const std::string idx = attr(line, "IDX");
      put(contigs, attr(line, "ID"), idx.empty() ? -1 : std::atoi(idx.c_str()));
    } else if (line.compare(0, 6, "#CHROM") == 0) {
      size_t a = 0;
      int col = 0;
      while (a <= line.size()) {
        size_t e = line.find('\t', a);
        if (e == std::string::npos) e = line.size();
        if (col >= 9) P.fam_iid.push_back(line.substr(a, e - a));
        ++col;
        a = e + 1;
      }
    }
  }
  P.n_file = static_cast<int>(P.fam_iid.size());
  P.bytes_per_snp = (P.n_file + 3) / 4;
  if (P.n_file == 0) die("BCF has no samples");
  P.dense = prefer_ds;
  if (prefer_ds) info("VCF: FORMAT/DS present -> use dosage field when available");
  int gt_key = -1, ds_key = -1;
  for (size_t k = 0; k < dict.size(); ++k) {
    if (dict[k] == "GT") gt_key = static_cast<int>(k);
    if (dict[k] == "DS") ds_key = static_cast<int>(k);
  }
  const int n = P.n_file;
  int64_t n_rec = 0;
  for (size_t off = 9 + l_text; off < text.size();) {
    BcfReader r(text, off);
    const uint32_t l_shared = r.u32(), l_indiv = r.u32();
    const size_t shared0 = r.at, indiv0 = shared0 + l_shared;
    off = indiv0 + l_indiv;
    if (off > text.size()) die("BCF record truncated");
    ++n_rec;
    const int32_t chrom_idx = static_cast<int32_t>(r.u32());
    const int32_t pos0 = static_cast<int32_t>(r.u32());
    r.u32();  // rlen
    r.u32();  // QUAL
    const uint32_t n_allele_info = r.u32(), n_fmt_sample = r.u32();
    const int n_allele = static_cast<int>(n_allele_info >> 16), n_info = static_cast<int>(n_allele_info & 0xFFFF);
    const int n_fmt = static_cast<int>(n_fmt_sample >> 24), n_smp = static_cast<int>(n_fmt_sample & 0xFFFFFF);
    std::string id = r.string_value();
    if (n_allele != 2) {  // not biallelic
      ++vi.n_multi;
      continue;
    }
    const std::string ref = r.string_value(), alt = r.string_value();
    r.skip_typed();  // FILTER
    for (int k = 0; k < n_info; ++k) {
      r.int_value();
      r.skip_typed();
    }
    if (r.at != indiv0) die("BCF shared block length mismatch");
    if (n_smp < n) die("VCF record with fewer sample columns than the header");
    // FORMAT arrays
    const char* gt = nullptr;
    const char* dsv = nullptr;
    int gt_t = 0, gt_c = 0, ds_t = 0, ds_c = 0;
    for (int k = 0; k < n_fmt; ++k) {
      const int64_t key = r.int_value();
      int t;
      int64_t c;
      r.desc(t, c);
      const size_t bytes = BcfReader::width(t) * static_cast<size_t>(c) * static_cast<size_t>(n_smp);
      r.need(bytes);
      if (key == gt_key) {
        gt = text.data() + r.at;
        gt_t = t;
        gt_c = static_cast<int>(c);
      } else if (key == ds_key) {
        dsv = text.data() + r.at;
        ds_t = t;
        ds_c = static_cast<int>(c);
      }
      r.at += bytes;
    }
    const bool use_ds = prefer_ds && ds_float && dsv != nullptr && ds_t == 5 && ds_c >= 1;
    if (!use_ds && (gt == nullptr || gt_c < 1 || BcfReader::width(gt_t) == 0 || gt_t == 5 || gt_t == 7)) continue;
    if (use_ds && !said_ds) {
      info("VCF: using FORMAT/DS dosages");
      said_ds = true;
    }
    if (chrom_idx < 0 || static_cast<size_t>(chrom_idx) >= contigs.size()) die("BCF CHROM index outside the contigs");
    const std::string chrom = contigs[static_cast<size_t>(chrom_idx)];
    const bool hap = haploid_chrom(chrom);
    std::vector<uint8_t> row(P.dense ? 0 : static_cast<size_t>(P.bytes_per_snp), 0);
    std::vector<float> drow(P.dense ? static_cast<size_t>(n) : 0);
    std::vector<int32_t> hap_calls;
    for (int i = 0; i < n; ++i) {
      if (use_ds) {
        // the reference reads the flattened float array at the sample's column
        uint32_t bits;
        std::memcpy(&bits, dsv + 4 * static_cast<size_t>(i), 4);
        float v;
        std::memcpy(&v, &bits, 4);
        drow[static_cast<size_t>(i)] = (bits == 0x7F800001u || bits == 0x7F800002u || !std::isfinite(v))
                                           ? std::numeric_limits<float>::quiet_NaN()
                                           : v;
        continue;
      }
      const size_t w = BcfReader::width(gt_t);
      const char* g = gt + w * static_cast<size_t>(gt_c) * i;
      const int32_t a0 = widen(g, gt_t);
      const int32_t a1 = gt_c > 1 ? widen(g + w, gt_t) : INT32_MIN + 1;
      const auto is_missing = [](int32_t v) { return (v >> 1) == 0 || v == INT32_MIN; };
      bool miss = is_missing(a0) || a0 == INT32_MIN + 1;
      if (!miss && gt_c > 1 && a1 != INT32_MIN + 1 && a1 != INT32_MIN) miss = is_missing(a1);
      int d = -1;
      bool haploid = false;
      if (!miss) {
        d = (a0 >> 1) - 1;
        int na = 1;
        if (gt_c > 1 && a1 != INT32_MIN + 1 && a1 != INT32_MIN) {
          d += (a1 >> 1) - 1;
          ++na;
        }
        if ((a0 >> 1) - 1 > 1 || (na == 2 && (a1 >> 1) - 1 > 1))
          die("VCF GT allele index beyond the single ALT allele");
        haploid = na == 1;
      }
      if (P.dense) {
        drow[static_cast<size_t>(i)] = d < 0 ? std::numeric_limits<float>::quiet_NaN() : static_cast<float>(d);
      } else {
        const uint32_t code = d < 0 ? 1u : (d == 2 ? 0u : (d == 1 ? 2u : 3u));
        row[static_cast<size_t>(i >> 2)] |= static_cast<uint8_t>(code << ((i & 3) * 2));
      }
      if (d >= 0 && haploid && !hap) hap_calls.push_back(i);
    }
    P.chrom.push_back(chrom);
    P.pos.push_back(static_cast<int64_t>(pos0) + 1);
    P.id.push_back(id == "." ? std::string() : id);
    P.a2.push_back(ref);
    P.a1.push_back(alt);
    P.rows.insert(P.rows.end(), row.begin(), row.end());
    P.ds.insert(P.ds.end(), drow.begin(), drow.end());
    vi.hap_chrom.push_back(hap ? 1 : 0);
    vi.hap_calls.push_back(std::move(hap_calls));
  }
  if (vi.n_multi > 0)
    info("VCF multi-allelic sites skipped (biallelic only): " + std::to_string(vi.n_multi));
  info("VCF: " + std::to_string(P.chrom.size()) + " biallelic records of " + std::to_string(n_rec) + " on " +
       std::to_string(P.n_file) + " samples");
  return P;
}

}  // namespace

Plink read_vcf(const std::string& path, VcfInfo& vi, const std::function<eqtl_ctx*()>& get_ctx) {
  Trace tr;
  const std::string text = read_all(path);
  tr.mark("VCF: read and inflate " + std::to_string(text.size()) + " bytes");
  if (text.empty()) die("empty VCF: " + path);
  if (text.compare(0, 3, "BCF") == 0) return read_bcf_records(text, vi);
  Plink P;
  bool have_header = false;
  int64_t n_rec = 0;
  bool prefer_ds = false, ds_float = false, said_ds = false;
  // records kept: where their sample columns lie, the FORMAT positions used
  std::vector<int64_t> beg, end;
  std::vector<int32_t> gt_at_v, ds_at_v;
  const char* T = text.data();
  const size_t N = text.size();
  for (size_t ls = 0; ls < N;) {
    const void* nl = std::memchr(T + ls, '\n', N - ls);
    size_t le = nl ? static_cast<const char*>(nl) - T : N;
    const size_t next = nl ? le + 1 : N;
    if (le > ls && T[le - 1] == '\r') --le;
    if (le == ls) {
      ls = next;
      continue;
    }
    if (T[ls] == '#') {
      const std::string line(T + ls, le - ls);
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
      ls = next;
      continue;
    }
    if (!have_header) die("VCF record before the #CHROM header line: " + path);
    ++n_rec;
    // the nine fixed columns
    size_t f[10];
    f[0] = ls;
    int nf = 1;
    for (size_t a = ls; nf < 10;) {
      const void* tb = a < le ? std::memchr(T + a, '\t', le - a) : nullptr;
      if (!tb) break;
      a = static_cast<const char*>(tb) - T + 1;
      f[nf++] = a;
    }
    if (nf < 10) die("VCF record with fewer sample columns than the header");
    auto col = [&](int k) { return std::string(T + f[k], f[k + 1] - 1 - f[k]); };
    const std::string alt = col(4);
    if (alt == "." || alt.find(',') != std::string::npos) {  // not biallelic (n_allele != 2)
      ++vi.n_multi;
      ls = next;
      continue;
    }
    int gt_at = -1, ds_at = -1;
    {
      int k = 0;
      size_t s = 0;
      const std::string fmt = col(8);
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
    if (!use_ds && gt_at < 0) {  // no genotypes in this record
      ls = next;
      continue;
    }
    if (use_ds && !said_ds) {
      info("VCF: using FORMAT/DS dosages");
      said_ds = true;
    }
    const std::string chrom = col(0);
    P.chrom.push_back(chrom);
    P.pos.push_back(std::stoll(col(1)));
    const std::string id = col(2);
    P.id.push_back(id == "." ? std::string() : id);
    P.a2.push_back(col(3));  // REF
    P.a1.push_back(alt);     // ALT, the counted allele
    vi.hap_chrom.push_back(haploid_chrom(chrom) ? 1 : 0);
    beg.push_back(static_cast<int64_t>(f[9]));
    end.push_back(static_cast<int64_t>(le));
    gt_at_v.push_back(gt_at);
    ds_at_v.push_back(use_ds ? ds_at : -1);
    ls = next;
  }
  if (!have_header) die("VCF without a #CHROM header line: " + path);
  tr.mark("VCF: fixed columns of " + std::to_string(n_rec) + " records");
  // the calls, on the device, in batches of at most 1 GiB of text
  const int64_t R = static_cast<int64_t>(beg.size());
  const int n = P.n_file;
  const int64_t bpr = P.bytes_per_snp, hbr = (n + 7) / 8;
  if (P.dense) P.ds.resize(static_cast<size_t>(R) * n);
  else P.rows.assign(static_cast<size_t>(R * bpr), 0);
  std::vector<uint8_t> hap(static_cast<size_t>(R * hbr), 0), flag(static_cast<size_t>(R), 0);
  eqtl_ctx* ctx = R > 0 ? get_ctx() : nullptr;
  tr.mark("VCF: device opened");
  for (int64_t r0 = 0; r0 < R;) {
    int64_t r1 = r0 + 1;
    while (r1 < R && end[r1] - beg[r0] <= (int64_t(1) << 30) && (r1 - r0) * n < (int64_t(1) << 27)) ++r1;
    const int64_t base = beg[r0];
    std::vector<int64_t> b(beg.begin() + r0, beg.begin() + r1), e(end.begin() + r0, end.begin() + r1);
    for (auto& v : b) v -= base;
    for (auto& v : e) v -= base;
    const int rc = eqtl_vcf_parse(ctx, T + base, end[r1 - 1] - base, b.data(), e.data(), gt_at_v.data() + r0,
                                  ds_at_v.data() + r0, r1 - r0, n, P.dense ? 1 : 0,
                                  P.dense ? nullptr : P.rows.data() + r0 * bpr,
                                  P.dense ? P.ds.data() + r0 * n : nullptr, hap.data() + r0 * hbr, flag.data() + r0);
    if (rc != EQTL_OK) die(std::string("VCF parse on the device: ") + eqtl_last_error(ctx));
    r0 = r1;
  }
  tr.mark("VCF: calls parsed on the device");
  vi.hap_calls.assign(static_cast<size_t>(R), {});
  for (int64_t r = 0; r < R; ++r) {
    if (flag[r] == 1) die("VCF record with fewer sample columns than the header");
    const bool use_ds = ds_at_v[r] >= 0;
    if (flag[r] == 2) {
      // a call outside the device parser's fast paths: this record on the host
      const char* s0 = T + beg[r];
      size_t a = 0;
      const size_t len = static_cast<size_t>(end[r] - beg[r]);
      uint8_t* row = P.dense ? nullptr : P.rows.data() + r * bpr;
      if (row) std::fill(row, row + bpr, 0);
      std::fill(hap.begin() + r * hbr, hap.begin() + (r + 1) * hbr, 0);
      for (int i = 0; i < n; ++i) {
        size_t b = a;
        while (b < len && s0[b] != '\t') ++b;
        const char* s = s0 + a;
        const size_t sl = b - a;
        a = b + 1;
        size_t p0 = 0, p1 = 0;
        if (use_ds) {
          P.ds[static_cast<size_t>(r) * n + i] =
              subfield(s, sl, ds_at_v[r], p0, p1) ? parse_ds(s + p0, p1 - p0) : std::numeric_limits<float>::quiet_NaN();
          continue;
        }
        bool haploid = false;
        const int d = (subfield(s, sl, gt_at_v[r], p0, p1) && p1 > p0) ? parse_gt(s + p0, p1 - p0, haploid) : -1;
        if (P.dense) {
          P.ds[static_cast<size_t>(r) * n + i] = d < 0 ? std::numeric_limits<float>::quiet_NaN() : static_cast<float>(d);
        } else {
          const uint32_t code = d < 0 ? 1u : (d == 2 ? 0u : (d == 1 ? 2u : 3u));
          row[i >> 2] |= static_cast<uint8_t>(code << ((i & 3) * 2));
        }
        if (d >= 0 && haploid) hap[static_cast<size_t>(r * hbr + (i >> 3))] |= static_cast<uint8_t>(1u << (i & 7));
      }
    }
    if (use_ds || vi.hap_chrom[static_cast<size_t>(r)]) continue;  // ploidy from the chromosome
    for (int i = 0; i < n; ++i)
      if (hap[static_cast<size_t>(r * hbr + (i >> 3))] >> (i & 7) & 1u) vi.hap_calls[static_cast<size_t>(r)].push_back(i);
  }
  tr.mark("VCF: host fallbacks and haploid calls");
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
