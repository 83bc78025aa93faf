// Test infrastructure only: replaces src/vcf_session.cpp, which needs htslib
// 1.24 (an empty submodule in the reference tree). The oracle build reads
// PLINK .bed only; every VCF entry point stops with the reference's own
// error path (die -> "[E] ..." and exit 1).
#include "eqtl/vcf_session.hpp"
#include "eqtl/util.hpp"

namespace eqtl {
static void no_vcf() { die("VCF input is not available in this oracle build (htslib absent); use -b/--bfile"); }
VcfSession::~VcfSession() {}
void VcfSession::set_threads(int) {}
void VcfSession::open(const std::string&) { no_vcf(); }
void VcfSession::set_sample_order(const std::vector<std::string>&) { no_vcf(); }
void VcfSession::for_each_snp(const MissPolicy&, double, const std::function<bool(const SnpRec&)>&) { no_vcf(); }
void VcfSession::for_each_snp_region(const std::string&, int64_t, int64_t, const MissPolicy&, double,
                                     const std::function<bool(const SnpRec&)>&) { no_vcf(); }
std::vector<SnpRec> VcfSession::load_all(const MissPolicy&, double, int) { no_vcf(); return {}; }
std::vector<SnpRec> VcfSession::load_region(const std::string&, int64_t, int64_t, const MissPolicy&, double) {
  no_vcf();
  return {};
}
}  // namespace eqtl
