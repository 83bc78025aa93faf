"""Maps a reference `eqtl` argv (as recorded in tests/golden/*/manifest.json)
onto the oracle driver's Options."""
from __future__ import annotations

import os

import driver


def options_from_argv(argv, case_dir: str) -> driver.Options:
    o = driver.Options(bfile="", pheno="")
    it = iter(range(len(argv)))
    i = 0
    path = lambda v: os.path.join(case_dir, v)
    while i < len(argv):
        a = argv[i]
        v = argv[i + 1] if i + 1 < len(argv) else None
        step = 2
        if a in ("-b", "--bfile"):
            o.bfile = path(v)
        elif a in ("-e", "--pheno"):
            o.pheno = path(v)
        elif a in ("-g", "--gff"):
            o.gff = path(v)
        elif a in ("-c", "--covar"):
            o.covar = path(v)
        elif a in ("-k", "--grm"):
            o.grm = path(v)
        elif a == "--model":
            o.out_models = tuple(v.split(","))
        elif a in ("-m", "--mode"):
            o.mode = "gw" if v == "gwas" else v
        elif a in ("-w", "--window"):
            o.window = int(v)
        elif a == "--pval-cis":
            o.pval_cis = float(v)
        elif a == "--pval-trans":
            o.pval_trans = float(v)
        elif a == "--miss-hand":
            o.miss_hand = v
        elif a == "--max-miss":
            o.max_miss = float(v)
        elif a == "--maf":
            o.maf = float(v)
        elif a == "--perm":
            o.perm = int(v)
        elif a == "--perm-trans-thr":
            o.perm_trans_thr = float(v)
        elif a == "--perm-trans-top":
            o.perm_trans_top = int(v)
        elif a == "--seed":
            o.seed = int(v)
        elif a == "--pheno-norm":
            o.pheno_norm = v
        elif a in ("-t", "--thread", "--threads"):
            o.threads = int(v)
        elif a == "--fast":
            o.fast = True
            step = 1
        elif a == "--disable-beta-approx":
            o.disable_beta_approx = True
            step = 1
        elif a == "--make-grm":
            step = 1
        elif a in ("-o", "--out"):
            pass
        else:
            raise ValueError(f"unmapped flag {a}")
        i += step
    return o
