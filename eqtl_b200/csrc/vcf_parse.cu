// VCF sample columns parsed on the device: the GT (or FORMAT/DS) subfield of
// every call of a batch of records (VcfSession::parse_record's per-sample
// loop, src/vcf_session.cpp:193-258), from the decompressed text.
//
// The host splits the text into records and reads the nine fixed columns;
// per record it passes where the sample columns begin and end, which FORMAT
// subfield holds GT and which DS (-1: absent / not used). Then
//   vcf_starts_kernel  one warp per record finds the n_file sample columns:
//                      32 bytes per step, tab positions by ballot, the k-th
//                      tab starting sample k + 1;
//   vcf_calls_kernel   one thread per record and 8 samples parses the calls:
//                      GT -> ALT count (missing if either of the first two
//                      alleles is '.'), haploid when one allele is present;
//                      DS -> the first number of the subfield by the exact
//                      decimal fast path (at most 15 significant digits,
//                      |decimal exponent| <= 22: one correctly rounded
//                      multiply or divide, then rounded to FP32, as strtod
//                      and the cast give); "." or an absent subfield is
//                      missing.
// Outputs per record: 2-bit .bed codes (00 = 2 ALT, 10 = 1, 11 = 0,
// 01 = missing) or FP32 dosages (NaN = missing), one bit per call for a
// haploid GT call, and a flag: 1 when the record has fewer sample columns
// than the header, 2 when a call is outside the fast paths (a DS value in
// another notation, a GT with an allele index above 1 or malformed); the
// host parses flagged records itself. Every read stays inside the record's
// [begin, end).
#include <algorithm>

#include "internal.hpp"

namespace eqtl {
namespace {

__global__ void vcf_starts_kernel(const char* __restrict__ text, const int64_t* __restrict__ beg,
                                  const int64_t* __restrict__ end, int64_t R, int n_file, int64_t* starts,
                                  uint8_t* flag) {
  const int lane = threadIdx.x & 31;
  const int64_t r = static_cast<int64_t>(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= R) return;
  const int64_t b = beg[r], e = end[r];
  int64_t* st = starts + r * n_file;
  if (lane == 0) st[0] = b;
  int found = 0;  // tabs seen: sample `found` is the last one started
  for (int64_t pos = b; pos < e && found < n_file - 1; pos += 32) {
    const bool tab = pos + lane < e && text[pos + lane] == '\t';
    const unsigned m = __ballot_sync(0xffffffffu, tab);
    if (tab) {
      const int k = found + __popc(m & ((1u << lane) - 1u)) + 1;
      if (k < n_file) st[k] = pos + lane + 1;
    }
    found += __popc(m);
  }
  if (lane == 0 && found < n_file - 1) flag[r] = 1;
}

__device__ __forceinline__ bool is_digit(char c) { return c >= '0' && c <= '9'; }

// The first number of a DS subfield [p, q): NaN for "." or empty; false when
// the text is outside the exact fast path.
__device__ bool parse_ds_fast(const char* __restrict__ t, int64_t p, int64_t q, float& out) {
  const double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                             1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};
  for (int64_t i = p; i < q; ++i)
    if (t[i] == ',') {
      q = i;
      break;
    }
  if (q == p || (q == p + 1 && t[p] == '.')) {
    out = __int_as_float(0x7fc00000);
    return true;
  }
  int64_t i = p;
  bool neg = false;
  if (t[i] == '+' || t[i] == '-') {
    neg = t[i] == '-';
    ++i;
  }
  unsigned long long mant = 0;
  int sig = 0, frac = 0, digits = 0;
  bool dot = false;
  for (; i < q; ++i) {
    const char c = t[i];
    if (is_digit(c)) {
      ++digits;
      if (mant == 0 && c == '0') {
        if (dot) ++frac;  // leading zeros after the point
        continue;
      }
      if (++sig > 15) return false;
      mant = mant * 10 + static_cast<unsigned>(c - '0');
      if (dot) ++frac;
    } else if (c == '.' && !dot) {
      dot = true;
    } else {
      break;
    }
  }
  if (digits == 0) return false;
  int ex = 0;
  if (i < q && (t[i] == 'e' || t[i] == 'E')) {
    ++i;
    bool eneg = false;
    if (i < q && (t[i] == '+' || t[i] == '-')) {
      eneg = t[i] == '-';
      ++i;
    }
    int ed = 0;
    for (; i < q && is_digit(t[i]); ++i) {
      if (++ed > 3) return false;
      ex = ex * 10 + (t[i] - '0');
    }
    if (ed == 0) return false;
    if (eneg) ex = -ex;
  }
  if (i != q) return false;  // trailing text: leave it to the host
  const int e10 = ex - frac;
  double v = static_cast<double>(mant);
  if (mant != 0) {
    if (e10 > 22 || e10 < -22) return false;
    v = e10 >= 0 ? v * kPow10[e10] : v / kPow10[-e10];
  }
  if (neg) v = -v;
  const float f = static_cast<float>(v);
  out = isfinite(f) ? f : __int_as_float(0x7fc00000);
  return true;
}

// GT of [p, q): ALT count or -1 missing; haploid when one allele is
// present; false when malformed or an allele index is above 1.
__device__ bool parse_gt_fast(const char* __restrict__ t, int64_t p, int64_t q, int& d, bool& haploid) {
  int al[2] = {-2, -2};
  int na = 0;
  int64_t i = p;
  while (i < q && na < 2) {
    if (t[i] == '.') {
      al[na++] = -1;
      ++i;
    } else if (is_digit(t[i])) {
      int v = 0;
      while (i < q && is_digit(t[i])) {
        v = 10 * v + (t[i] - '0');
        if (v > 1000) return false;
        ++i;
      }
      al[na++] = v;
    } else {
      return false;
    }
    if (i < q && (t[i] == '/' || t[i] == '|')) ++i;
    else break;
  }
  haploid = false;
  if (na == 0 || al[0] == -1 || al[1] == -1) {
    d = -1;
    return true;
  }
  if (al[0] > 1 || al[1] > 1) return false;
  haploid = al[1] == -2;
  d = haploid ? al[0] : al[0] + al[1];
  return true;
}

__global__ void vcf_calls_kernel(const char* __restrict__ text, const int64_t* __restrict__ end,
                                 const int64_t* __restrict__ starts, const int32_t* __restrict__ gt_at,
                                 const int32_t* __restrict__ ds_at, int64_t R, int n_file, int dense,
                                 uint8_t* codes, int64_t bpr, float* ds, uint8_t* hap, int64_t hbr, uint8_t* flag) {
  const int groups = (n_file + 7) / 8;
  const int64_t total = R * groups;
  for (int64_t w = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; w < total;
       w += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t r = w / groups;
    const int grp = static_cast<int>(w - r * groups);
    if (flag[r] == 1) continue;  // too few columns: the host reports it
    const int64_t e = end[r];
    const int use_ds = ds_at[r] >= 0;
    const int sub = use_ds ? ds_at[r] : gt_at[r];
    uint32_t code16 = 0;  // 8 codes of 2 bits
    uint32_t hbits = 0;
    bool bad = false;
    for (int t = 0; t < 8; ++t) {
      const int smp = grp * 8 + t;
      if (smp >= n_file) break;
      const int64_t s = starts[r * n_file + smp];
      int64_t f = s;  // end of the sample column
      while (f < e && text[f] != '\t') ++f;
      // the sub-th ':'-separated subfield
      int64_t p = s;
      bool have = true;
      for (int k = 0; k < sub && have; ++k) {
        while (p < f && text[p] != ':') ++p;
        if (p < f) ++p;
        else have = false;
      }
      int64_t q = p;
      while (have && q < f && text[q] != ':') ++q;
      if (use_ds) {
        float v = __int_as_float(0x7fc00000);
        if (have && !parse_ds_fast(text, p, q, v)) bad = true;
        ds[r * n_file + smp] = v;
        continue;
      }
      int d = -1;
      bool h = false;
      if (have && q > p && !parse_gt_fast(text, p, q, d, h)) bad = true;
      if (dense) ds[r * n_file + smp] = d < 0 ? __int_as_float(0x7fc00000) : static_cast<float>(d);
      const uint32_t c = d < 0 ? 1u : (d == 2 ? 0u : (d == 1 ? 2u : 3u));
      code16 |= c << (2 * t);
      if (d >= 0 && h) hbits |= 1u << t;
    }
    if (bad) flag[r] = 2;
    if (!use_ds && !dense) {
      const int64_t o = r * bpr + 2 * static_cast<int64_t>(grp);
      codes[o] = static_cast<uint8_t>(code16 & 0xFFu);
      if (2 * grp + 1 < bpr) codes[o + 1] = static_cast<uint8_t>(code16 >> 8);
    }
    if (!use_ds) hap[r * hbr + grp] = static_cast<uint8_t>(hbits);
  }
}

}  // namespace

void vcf_parse(eqtl_ctx* ctx, const char* text, int64_t text_len, const int64_t* beg, const int64_t* end,
               const int32_t* gt_at, const int32_t* ds_at, int64_t R, int n_file, int dense, uint8_t* codes_out,
               float* ds_out, uint8_t* hap_out, uint8_t* flag_out) {
  EQTL_CHECK(R >= 0 && n_file > 0 && text_len >= 0, EQTL_E_ARG, "vcf_parse: bad sizes");
  for (int64_t r = 0; r < R; ++r)
    EQTL_CHECK(beg[r] >= 0 && beg[r] <= end[r] && end[r] <= text_len, EQTL_E_ARG, "vcf_parse: record outside text");
  if (R == 0) return;
  cudaStream_t st = ctx->stream;
  const int64_t bpr = (n_file + 3) / 4, hbr = (n_file + 7) / 8;
  DevBuf<char> t;
  DevBuf<int64_t> b, e, starts;
  DevBuf<int32_t> g, d;
  DevBuf<uint8_t> codes, hap, flag;
  DevBuf<float> ds;
  t.upload(text, static_cast<size_t>(text_len), st);
  b.upload(beg, static_cast<size_t>(R), st);
  e.upload(end, static_cast<size_t>(R), st);
  g.upload(gt_at, static_cast<size_t>(R), st);
  d.upload(ds_at, static_cast<size_t>(R), st);
  starts.alloc(static_cast<size_t>(R) * n_file);
  flag.alloc(static_cast<size_t>(R));
  flag.zero(st);
  hap.alloc(static_cast<size_t>(R * hbr));
  hap.zero(st);
  if (!dense) codes.alloc(static_cast<size_t>(R * bpr));
  if (dense) ds.alloc(static_cast<size_t>(R) * n_file);
  ctx->launches += 2;
  vcf_starts_kernel<<<static_cast<unsigned>((R + 7) / 8), 256, 0, st>>>(t.p, b.p, e.p, R, n_file, starts.p, flag.p);
  const int64_t work = R * ((n_file + 7) / 8);
  vcf_calls_kernel<<<static_cast<unsigned>(std::min<int64_t>((work + 255) / 256, 148 * 64)), 256, 0, st>>>(
      t.p, e.p, starts.p, g.p, d.p, R, n_file, dense, codes.p, bpr, ds.p, hap.p, hbr, flag.p);
  EQTL_CUDA(cudaGetLastError());
  if (!dense) codes.download(codes_out, static_cast<size_t>(R * bpr), st);
  if (dense) ds.download(ds_out, static_cast<size_t>(R) * n_file, st);
  hap.download(hap_out, static_cast<size_t>(R * hbr), st);
  flag.download(flag_out, static_cast<size_t>(R), st);
  EQTL_CUDA(cudaStreamSynchronize(st));
}

}  // namespace eqtl
