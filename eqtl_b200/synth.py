"""Seeded synthetic eQTL inputs (PLINK .bed/.bim/.fam, phenotype and covariate
TSVs, GFF3 genes) with the shapes and value distributions of the benchmark
workloads.

No public data set ships with the reference, so every parity case and every
benchmark input is generated here from a fixed seed:

* genotypes: HWE dosages (A1 allele counts 0/1/2) at per-SNP allele frequency
  drawn from U(maf_lo, maf_hi), MCAR missingness at ``miss_rate``; optional
  family structure (founder haplotypes, siblings by Mendelian transmission)
  so the GRM has real relatedness;
* phenotypes: either N(0,1) noise plus planted effects (LM shapes), or a
  polygenic term with per-gene heritability h2 ~ U(0, h2_max) drawn from the
  genotype covariance (LMM shapes);
* covariates: N(0,1) columns, part of which leak into Y.

File formats follow the ones the reference reads: PLINK1 SNP-major .bed
(src/plink_bed.cpp:187-212, LUT :221-224), whitespace .bim/.fam
(:26-160), tab phenotype matrix with a sample column (src/pheno.cpp:17-75),
covariates (src/pheno.cpp:89-196) and GFF3 `gene` features
(src/annot.cpp:26-71).
"""
from __future__ import annotations

import dataclasses
import os
from typing import Optional, Sequence

import numpy as np

# 2-bit PLINK codes indexed by dosage (A1 count); -1 (missing) -> 0b01.
_CODE_OF_DOSAGE = {2: 0b00, 1: 0b10, 0: 0b11, -1: 0b01}


@dataclasses.dataclass
class Genotypes:
    codes: np.ndarray          # int8 [m, n]; 0/1/2 = A1 count, -1 = missing
    chrom: list                # per SNP chromosome name
    pos: np.ndarray            # int64 [m]
    ids: list                  # per SNP id
    a1: list
    a2: list
    samples: list              # per sample IID
    af: np.ndarray             # generating allele frequency per SNP


def pack_bed_rows(codes: np.ndarray) -> np.ndarray:
    """int8 dosage codes [m, n] -> uint8 SNP-major .bed rows [m, ceil(n/4)]."""
    m, n = codes.shape
    lut = np.zeros(256, dtype=np.uint8)
    for d, c in _CODE_OF_DOSAGE.items():
        lut[d & 0xFF] = c
    two = lut[codes.astype(np.int16) & 0xFF]
    nb = (n + 3) // 4
    pad = np.zeros((m, nb * 4), dtype=np.uint8)
    pad[:, :n] = two
    # padding samples decode as A1/A1 (00); readers ignore them.
    q = pad.reshape(m, nb, 4)
    return (q[:, :, 0] | (q[:, :, 1] << 2) | (q[:, :, 2] << 4) | (q[:, :, 3] << 6)).astype(np.uint8)


def hwe_codes(rng: np.random.Generator, n: int, m: int, maf_lo: float, maf_hi: float,
              miss_rate: float, af: Optional[np.ndarray] = None) -> tuple:
    if af is None:
        af = rng.uniform(maf_lo, maf_hi, size=m)
    # random orientation so A1 is the minor allele only half of the time
    flip = rng.random(m) < 0.5
    af = np.where(flip, 1.0 - af, af)
    codes = rng.binomial(2, af[:, None], size=(m, n)).astype(np.int8)
    if miss_rate > 0:
        codes[rng.random((m, n)) < miss_rate] = -1
    return codes, af


def family_codes(rng: np.random.Generator, m: int, n_fam: int, fam_size: int, n_unrel: int,
                 maf_lo: float, maf_hi: float, miss_rate: float) -> tuple:
    """Families of `fam_size` siblings from 2 founders each, plus unrelated
    samples. Returns int8 codes [m, n_fam*fam_size + n_unrel]."""
    af = rng.uniform(maf_lo, maf_hi, size=m)
    flip = rng.random(m) < 0.5
    af = np.where(flip, 1.0 - af, af)
    n = n_fam * fam_size + n_unrel
    codes = np.empty((m, n), dtype=np.int8)
    col = 0
    for _ in range(n_fam):
        # founder haplotypes [2 parents, 2 haplotypes, m]
        hap = (rng.random((2, 2, m)) < af[None, None, :]).astype(np.int8)
        for _ in range(fam_size):
            pick_p = rng.integers(0, 2, size=m)
            pick_m = rng.integers(0, 2, size=m)
            codes[:, col] = hap[0, pick_p, np.arange(m)] + hap[1, pick_m, np.arange(m)]
            col += 1
    if n_unrel:
        codes[:, col:] = rng.binomial(2, af[:, None], size=(m, n_unrel)).astype(np.int8)
    if miss_rate > 0:
        codes[rng.random((m, n)) < miss_rate] = -1
    return codes, af


def layout_snps(rng: np.random.Generator, m: int, n_chrom: int, chrom_len: int,
                chrom_prefix: str = "") -> tuple:
    """Uniform positions, sorted within chromosome blocks (the .bim order the
    reference requires, src/plink_bed.cpp:143-159)."""
    per = np.full(n_chrom, m // n_chrom)
    per[: m % n_chrom] += 1
    chrom, pos = [], []
    for c in range(n_chrom):
        p = np.sort(rng.choice(np.arange(1, chrom_len + 1), size=per[c], replace=False))
        chrom += [f"{chrom_prefix}{c + 1}"] * per[c]
        pos.append(p)
    return chrom, np.concatenate(pos).astype(np.int64)


def make_genotypes(seed: int, n: int, m: int, *, n_chrom: int = 5, chrom_len: int = 20_000_000,
                   maf_lo: float = 0.05, maf_hi: float = 0.5, miss_rate: float = 0.01,
                   family: Optional[tuple] = None) -> Genotypes:
    rng = np.random.default_rng(seed)
    if family is None:
        codes, af = hwe_codes(rng, n, m, maf_lo, maf_hi, miss_rate)
    else:
        n_fam, fam_size, n_unrel = family
        assert n_fam * fam_size + n_unrel == n
        codes, af = family_codes(rng, m, n_fam, fam_size, n_unrel, maf_lo, maf_hi, miss_rate)
    chrom, pos = layout_snps(rng, m, n_chrom, chrom_len)
    ids = [f"rs{i + 1}" for i in range(m)]
    bases = np.array(list("ACGT"))
    a1i = rng.integers(0, 4, size=m)
    a2i = (a1i + rng.integers(1, 4, size=m)) % 4
    samples = [f"S{i + 1:05d}" for i in range(n)]
    return Genotypes(codes, chrom, pos, ids, list(bases[a1i]), list(bases[a2i]), samples, af)


def write_plink(prefix: str, g: Genotypes) -> None:
    os.makedirs(os.path.dirname(prefix) or ".", exist_ok=True)
    with open(prefix + ".fam", "w") as f:
        for s in g.samples:
            f.write(f"{s} {s} 0 0 0 -9\n")
    with open(prefix + ".bim", "w") as f:
        for c, i, p, a1, a2 in zip(g.chrom, g.ids, g.pos, g.a1, g.a2):
            f.write(f"{c}\t{i}\t0\t{int(p)}\t{a1}\t{a2}\n")
    rows = pack_bed_rows(g.codes)
    with open(prefix + ".bed", "wb") as f:
        f.write(bytes([0x6C, 0x1B, 0x01]))
        f.write(rows.tobytes())


def imputed_dosage(codes: np.ndarray) -> np.ndarray:
    """Mean-imputed float dosages (the values the scans test)."""
    d = codes.astype(np.float64)
    miss = codes < 0
    d[miss] = 0.0
    n_ok = (~miss).sum(1)
    mu = d.sum(1) / np.maximum(n_ok, 1)
    d[miss] = np.broadcast_to(mu[:, None], d.shape)[miss]
    return d


def grm_like(codes: np.ndarray, n_snp: int, rng: np.random.Generator) -> np.ndarray:
    """Standardised genotypes of a random SNP subset; Z Z^T / k is the GRM."""
    m = codes.shape[0]
    pick = rng.choice(m, size=min(n_snp, m), replace=False)
    d = imputed_dosage(codes[pick])
    mu = d.mean(1, keepdims=True)
    p = mu / 2.0
    sd = np.sqrt(np.maximum(2 * p * (1 - p), 1e-12))
    return ((d - mu) / sd).T  # [n, k]


def make_pheno_lm(seed: int, g: Genotypes, n_genes: int, n_cov: int, *, cis_effects: bool,
                  gene_tss: Optional[np.ndarray] = None, gene_chrom: Optional[list] = None,
                  window: int = 1_000_000, n_trans: int = 0, beta_sd: float = 0.3,
                  cov_weight: float = 0.5) -> tuple:
    """Y = planted effects + cov_weight * sum(C) + N(0,1). Returns (Y [n, G], C [n, c])."""
    rng = np.random.default_rng(seed)
    n = len(g.samples)
    C = rng.standard_normal((n, n_cov))
    Y = rng.standard_normal((n, n_genes)) + cov_weight * C.sum(1, keepdims=True)
    dos = None
    if cis_effects and gene_tss is not None:
        chrom_arr = np.array(g.chrom)
        for j in range(n_genes):
            sel = np.nonzero((chrom_arr == gene_chrom[j]) & (np.abs(g.pos - gene_tss[j]) <= window))[0]
            if sel.size == 0:
                continue
            k = rng.integers(1, 4)
            pick = rng.choice(sel, size=min(k, sel.size), replace=False)
            d = imputed_dosage(g.codes[pick])
            Y[:, j] += (rng.normal(0.0, beta_sd, size=pick.size)[:, None] * d).sum(0)
    if n_trans:
        m = g.codes.shape[0]
        snps = rng.integers(0, m, size=n_trans)
        genes = rng.integers(0, n_genes, size=n_trans)
        d = imputed_dosage(g.codes[snps])
        for t in range(n_trans):
            Y[:, genes[t]] += rng.normal(0.0, beta_sd) * d[t]
    return Y, C


def make_pheno_lmm(seed: int, g: Genotypes, n_genes: int, n_cov: int, *, h2_max: float = 0.8,
                   n_poly_snps: int = 2000, cov_weight: float = 0.5, n_trans: int = 0,
                   beta_sd: float = 0.2) -> tuple:
    """y = sqrt(h2) u + sqrt(1-h2) e with u ~ N(0, GRM) drawn from standardised
    genotypes; h2 ~ U(0, h2_max) per gene."""
    rng = np.random.default_rng(seed)
    n = len(g.samples)
    Z = grm_like(g.codes, n_poly_snps, rng)
    k = Z.shape[1]
    h2 = rng.uniform(0.0, h2_max, size=n_genes)
    u = Z @ rng.standard_normal((k, n_genes)) / np.sqrt(k)
    e = rng.standard_normal((n, n_genes))
    Y = np.sqrt(h2)[None, :] * u + np.sqrt(1 - h2)[None, :] * e
    C = rng.standard_normal((n, n_cov))
    if n_cov:
        Y += cov_weight * C.sum(1, keepdims=True)
    if n_trans:
        m = g.codes.shape[0]
        snps = rng.integers(0, m, size=n_trans)
        genes = rng.integers(0, n_genes, size=n_trans)
        d = imputed_dosage(g.codes[snps])
        for t in range(n_trans):
            Y[:, genes[t]] += rng.normal(0.0, beta_sd) * d[t]
    return Y, C, h2


def make_pheno_counts(seed: int, g: Optional[Genotypes], n_genes: int, n_cov: int, *, n_trans: int = 0,
                      beta_sd: float = 0.3, cov_weight: float = 0.2, n: Optional[int] = None) -> tuple:
    """Negative-binomial counts (NB2, log link): log mu = b0 + cov_weight *
    sum(C) + planted SNP effects, b0 ~ U(0.5, 4), dispersion phi ~ U(0.05, 1)
    per gene, y ~ Poisson(Gamma(1/phi, phi mu)). Returns (Y [n, G], C [n, c]).
    Without genotypes (g None, n given) no SNP effects are planted."""
    rng = np.random.default_rng(seed)
    n = len(g.samples) if g is not None else n
    C = rng.standard_normal((n, n_cov))
    eta = rng.uniform(0.5, 4.0, n_genes)[None, :] + cov_weight * C.sum(1, keepdims=True)
    if n_trans and g is not None:
        m = g.codes.shape[0]
        snps = rng.integers(0, m, size=n_trans)
        genes = rng.integers(0, n_genes, size=n_trans)
        d = imputed_dosage(g.codes[snps])
        for t in range(n_trans):
            eta[:, genes[t]] += rng.normal(0.0, beta_sd) * (d[t] - d[t].mean())
    phi = rng.uniform(0.05, 1.0, n_genes)
    mu = np.exp(eta)
    lam = rng.gamma(1.0 / phi[None, :], phi[None, :] * mu)
    return rng.poisson(lam).astype(np.float64), C


def make_genes(seed: int, n_genes: int, chroms: Sequence[str], chrom_len: int,
               body: int = 1) -> tuple:
    """Genes with uniform TSS, strand +/- 50/50, body length `body` bp."""
    rng = np.random.default_rng(seed)
    gchrom = [chroms[i] for i in rng.integers(0, len(chroms), size=n_genes)]
    start = rng.integers(1, chrom_len - body, size=n_genes).astype(np.int64)
    end = start + body - 1
    strand = np.where(rng.random(n_genes) < 0.5, "+", "-")
    ids = [f"G{i + 1:05d}" for i in range(n_genes)]
    tss = np.where(strand == "-", end, start)
    return ids, gchrom, start, end, strand, tss


def _ds_text(v) -> str:
    return "." if not np.isfinite(v) else np.format_float_positional(np.float32(v), unique=True, trim="-")


def write_bgzf(path: str, text: str) -> None:
    """BGZF (blocked gzip, the SAM/VCF specifications' container): gzip
    members of at most 65,280 text bytes, each with the BC extra field giving
    the member's size, then the empty end-of-file member."""
    import struct
    import zlib
    data = text.encode() if isinstance(text, str) else bytes(text)
    with open(path, "wb") as f:
        for a in range(0, len(data), 65280):
            chunk = data[a:a + 65280]
            co = zlib.compressobj(6, zlib.DEFLATED, -15)
            comp = co.compress(chunk) + co.flush()
            f.write(struct.pack("<BBBBIBBHBBHH", 31, 139, 8, 4, 0, 0, 255, 6, 66, 67, 2, len(comp) + 25))
            f.write(comp)
            f.write(struct.pack("<II", zlib.crc32(chunk) & 0xFFFFFFFF, len(chunk)))
        f.write(bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000"))


def write_vcf(path: str, samples: Sequence[str], chrom: Sequence[str], pos: Sequence[int], ids: Sequence[str],
              ref: Sequence[str], alt: Sequence[str], dosage: np.ndarray, haploid: Optional[np.ndarray] = None,
              phased: bool = False, ds: Optional[np.ndarray] = None, ds_rows: Optional[np.ndarray] = None,
              bgzf: bool = False, ds_text=None) -> None:
    """VCF 4.2 with a GT field (gzip-compressed when `path` ends in .gz):
    dosage [m, n] = ALT allele count (-1 missing); haploid [m, n] marks calls
    written with one allele ("0", "1", "."). With `ds` [m, n] (NaN = ".") the
    header declares FORMAT/DS and the records where `ds_rows` is set (all by
    default) carry GT:DS, each DS value written as the shortest text that
    reads back as the same FP32 number (or as `ds_text(value)` gives it).
    bgzf: a .gz path is written as BGZF instead of one gzip member."""
    import gzip
    import io
    sep = "|" if phased else "/"
    gt_dip = {0: f"0{sep}0", 1: f"0{sep}1", 2: f"1{sep}1", -1: f".{sep}."}
    gt_hap = {0: "0", 1: "1", -1: "."}
    if ds is not None and ds_rows is None:
        ds_rows = np.ones(len(chrom), bool)
    fmt_ds = ds_text or _ds_text
    f = io.StringIO()
    if True:
        f.write("##fileformat=VCFv4.2\n")
        f.write('##FORMAT=<ID=GT,Number=1,Type=String,Description="Genotype">\n')
        if ds is not None:
            f.write('##FORMAT=<ID=DS,Number=A,Type=Float,Description="Estimated ALT dose, [P(0/1) + 2*P(1/1)]">\n')
        f.write("#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\t" + "\t".join(samples) + "\n")
        for r in range(len(chrom)):
            d = dosage[r]
            h = haploid[r] if haploid is not None else np.zeros(len(d), bool)
            calls = [gt_hap[int(v)] if hh else gt_dip[int(v)] for v, hh in zip(d, h)]
            fmt = "GT"
            if ds is not None and ds_rows[r]:
                fmt = "GT:DS"
                calls = [c + ":" + fmt_ds(v) for c, v in zip(calls, ds[r])]
            f.write(f"{chrom[r]}\t{int(pos[r])}\t{ids[r] or '.'}\t{ref[r]}\t{alt[r]}\t.\tPASS\t.\t{fmt}\t" +
                    "\t".join(calls) + "\n")
    text = f.getvalue()
    if path.endswith(".gz") and bgzf:
        write_bgzf(path, text)
    elif path.endswith(".gz"):
        with gzip.open(path, "wt") as g:
            g.write(text)
    else:
        with open(path, "w") as g:
            g.write(text)


def write_bcf(path: str, samples: Sequence[str], chrom: Sequence[str], pos: Sequence[int], ids: Sequence[str],
              ref: Sequence[str], alt: Sequence[str], dosage: np.ndarray, haploid: Optional[np.ndarray] = None,
              ds: Optional[np.ndarray] = None) -> None:
    """The genotypes of write_vcf as BCF2 (BGZF-compressed), laid out as the
    VCF specification's BCF2 section describes: the header text with its
    string dictionary (PASS, GT, DS) and contig list, then per record the
    shared fields (contig index, 0-based POS, ID, REF, ALT, FILTER PASS) and
    the FORMAT arrays: GT as int8 pairs ((allele + 1) << 1, 0 for '.', the
    vector-end byte 0x81 after a haploid call) and, with `ds`, DS as FP32
    (missing 0x7F800001)."""
    import struct
    contigs = list(dict.fromkeys(chrom))
    head = "##fileformat=VCFv4.2\n##FILTER=<ID=PASS,Description=\"All filters passed\">\n"
    head += '##FORMAT=<ID=GT,Number=1,Type=String,Description="Genotype">\n'
    if ds is not None:
        head += '##FORMAT=<ID=DS,Number=A,Type=Float,Description="Estimated ALT dose">\n'
    for c in contigs:
        head += f"##contig=<ID={c}>\n"
    head += "#CHROM\tPOS\tID\tREF\tALT\tQUAL\tFILTER\tINFO\tFORMAT\t" + "\t".join(samples) + "\n"
    hb = head.encode() + b"\0"

    def typed_str(t: str) -> bytes:
        e = t.encode()
        if len(e) < 15:
            return bytes([(len(e) << 4) | 7]) + e
        return bytes([(15 << 4) | 7, 0x11, len(e)]) + e if len(e) < 128 else \
            bytes([(15 << 4) | 7, 0x12]) + struct.pack("<h", len(e)) + e

    n = len(samples)
    out = bytearray(b"BCF\x02\x02" + struct.pack("<I", len(hb)) + hb)
    pairs = {0: (0, 0), 1: (0, 1), 2: (1, 1)}
    for r in range(len(chrom)):
        shared = struct.pack("<iiiIII", contigs.index(chrom[r]), int(pos[r]) - 1, len(ref[r]), 0x7F800001,
                             2 << 16, ((2 if ds is not None else 1) << 24) | n)
        shared += typed_str(ids[r] or ".") + typed_str(ref[r]) + typed_str(alt[r]) + bytes([0x11, 0])
        gt = bytearray()
        for i in range(n):
            d = int(dosage[r, i])
            h = haploid is not None and bool(haploid[r, i])
            if h:
                gt += bytes([0 if d < 0 else ((d + 1) << 1), 0x81])
            elif d < 0:
                gt += bytes([0, 0])
            else:
                a0, a1 = pairs[d]
                gt += bytes([(a0 + 1) << 1, (a1 + 1) << 1])
        indiv = bytes([0x11, 1, (2 << 4) | 1]) + bytes(gt)
        if ds is not None:
            vals = b"".join(struct.pack("<I", 0x7F800001) if not np.isfinite(v) else struct.pack("<f", v)
                            for v in ds[r])
            indiv += bytes([0x11, 2, (1 << 4) | 5]) + vals
        out += struct.pack("<II", len(shared), len(indiv)) + shared + indiv
    write_bgzf(path, bytes(out))


def write_tabix_header(vcf_path: str) -> None:
    """<vcf_path>.tbi holding a tabix index of no sequences (the magic and the
    VCF preset): enough for a reader that only checks that an index exists;
    a region query through it finds nothing."""
    import gzip
    import struct
    with gzip.open(vcf_path + ".tbi", "wb") as f:
        f.write(b"TBI\x01" + struct.pack("<8i", 0, 2, 1, 2, 0, ord("#"), 0, 0))


def write_pheno(path: str, samples: Sequence[str], genes: Sequence[str], Y: np.ndarray) -> None:
    with open(path, "w") as f:
        f.write("sample\t" + "\t".join(genes) + "\n")
        for i, s in enumerate(samples):
            f.write(s + "\t" + "\t".join(repr(float(v)) if np.isfinite(v) else "NA" for v in Y[i]) + "\n")


def write_covar(path: str, samples: Sequence[str], C: np.ndarray) -> None:
    with open(path, "w") as f:
        f.write("sample\t" + "\t".join(f"cov{j + 1}" for j in range(C.shape[1])) + "\n")
        for i, s in enumerate(samples):
            f.write(s + "\t" + "\t".join(repr(float(v)) for v in C[i]) + "\n")


def write_gff(path: str, ids, chrom, start, end, strand) -> None:
    with open(path, "w") as f:
        f.write("##gff-version 3\n")
        for i, c, s, e, st in zip(ids, chrom, start, end, strand):
            f.write(f"{c}\tsynth\tgene\t{int(s)}\t{int(e)}\t.\t{st}\t.\tID={i};Name={i}\n")


def _fast_codes(rng: np.random.Generator, mc: int, n: int, family: Optional[tuple], maf_lo: float,
                maf_hi: float, miss_rate: float) -> np.ndarray:
    """Vectorised float32 sampler for the large shapes: [mc, n] int8 codes."""
    af = rng.uniform(maf_lo, maf_hi, size=mc).astype(np.float32)
    af = np.where(rng.random(mc) < 0.5, 1.0 - af, af).astype(np.float32)[:, None]
    codes = np.empty((mc, n), dtype=np.int8)
    col = 0
    if family is not None:
        n_fam, fam_size, n_unrel = family
        # founder haplotypes [fam, parent, hap, snp] and the haplotype each
        # sibling inherits from each parent
        H = rng.random((n_fam, 2, 2, mc), dtype=np.float32) < af[None, None, None, :, 0]
        pick = rng.random((n_fam, fam_size, 2, mc), dtype=np.float32) < 0.5
        from_p = np.where(pick[:, :, 0], H[:, None, 0, 1], H[:, None, 0, 0])
        from_m = np.where(pick[:, :, 1], H[:, None, 1, 1], H[:, None, 1, 0])
        sib = (from_p.astype(np.int8) + from_m.astype(np.int8)).reshape(n_fam * fam_size, mc)
        codes[:, : n_fam * fam_size] = sib.T
        col = n_fam * fam_size
    if col < n:
        k = n - col
        codes[:, col:] = ((rng.random((mc, k), dtype=np.float32) < af).astype(np.int8) +
                          (rng.random((mc, k), dtype=np.float32) < af).astype(np.int8))
    if miss_rate > 0:
        codes[rng.random((mc, n), dtype=np.float32) < miss_rate] = -1
    return codes


def make_bed_rows_chunked(seed: int, n: int, m: int, *, family: Optional[tuple] = None, maf_lo: float = 0.01,
                          maf_hi: float = 0.5, miss_rate: float = 0.01, chunk: int = 32768,
                          keep_codes_every: int = 0) -> tuple:
    """Packed .bed rows [m, ceil(n/4)] generated in SNP chunks (bounded host
    memory for the large benchmark shapes). With family=(n_fam, fam_size,
    n_unrel) siblings inherit founder alleles by Mendelian transmission.
    Also returns int8 codes of every `keep_codes_every`-th SNP (for drawing
    polygenic phenotypes) and their indices."""
    rng = np.random.default_rng(seed)
    nb = (n + 3) // 4
    rows = np.empty((m, nb), dtype=np.uint8)
    kept_codes, kept_idx = [], []
    for s0 in range(0, m, chunk):
        mc = min(chunk, m - s0)
        codes = _fast_codes(rng, mc, n, family, maf_lo, maf_hi, miss_rate)
        rows[s0:s0 + mc] = pack_bed_rows(codes)
        if keep_codes_every:
            sel = np.arange((-s0) % keep_codes_every, mc, keep_codes_every)
            kept_codes.append(codes[sel])
            kept_idx.append(s0 + sel)
    if keep_codes_every:
        return rows, np.concatenate(kept_codes), np.concatenate(kept_idx)
    return rows, None, None


def polygenic_pheno(seed: int, codes_sub: np.ndarray, n_genes: int, h2_max: float = 0.8) -> tuple:
    """y = sqrt(h2) u + sqrt(1-h2) e, u ~ N(0, GRM of the given SNP subset)."""
    rng = np.random.default_rng(seed)
    d = imputed_dosage(codes_sub)
    mu = d.mean(1, keepdims=True)
    p = mu / 2.0
    sd = np.sqrt(np.maximum(2 * p * (1 - p), 1e-12))
    Z = ((d - mu) / sd).T
    k = Z.shape[1]
    n = Z.shape[0]
    h2 = rng.uniform(0.0, h2_max, size=n_genes)
    Y = np.empty((n, n_genes))
    for g0 in range(0, n_genes, 2048):
        g1 = min(n_genes, g0 + 2048)
        u = Z @ rng.standard_normal((k, g1 - g0)) / np.sqrt(k)
        e = rng.standard_normal((n, g1 - g0))
        Y[:, g0:g1] = np.sqrt(h2[g0:g1])[None, :] * u + np.sqrt(1 - h2[g0:g1])[None, :] * e
    return Y, h2
