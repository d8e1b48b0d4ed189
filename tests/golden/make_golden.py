"""Regenerate the golden fixtures of this directory from the reference tree.

* family.a3m / family_pssm.json: the reference's demo MSA and the PSSM it
  wrote for it (demo/family.a3m, demo/family.pssm; `sabertooth profile`
  output): pins the PSSM construction that builds PSSM query rows.
* v1_fixture.fa / v1_fixture_k2_v03.json: the reference's test database
  (tests/data/v1_fixture.fa) and the search output that its test
  `cli_db_equivalence.rs` requires the current code to reproduce
  (tests/data/v1_fixture_k2.v03.m8: every sequence against the database,
  BLOSUM62 11/1 with composition-bias correction and the scoring mask).

The m8 tables are stored as parsed records (query, target, alignment span,
E-value and bits as printed).

Run where the reference tree is present:
    python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def parse_m8(path):
    lines = open(path).read().splitlines()
    head = lines[0].split("\t")
    out = []
    for ln in lines[1:]:
        f = dict(zip(head, ln.split("\t")))
        out.append({"query": f["query"], "target": f["target"], "qstart": int(f["qstart"]), "qend": int(f["qend"]),
                    "tstart": int(f["tstart"]), "tend": int(f["tend"]), "evalue": f["evalue"], "bits": f["bits"]})
    return out


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py /path/to/reference")
    ref = sys.argv[1]
    shutil.copyfile(os.path.join(ref, "demo", "family.a3m"), os.path.join(HERE, "family.a3m"))
    lines = open(os.path.join(ref, "demo", "family.pssm")).read().splitlines()
    header = lines[0].split()
    letters = header[2:22]
    rows, neff, qres = [], [], []
    for ln in lines[1:]:
        tok = ln.split()
        qres.append(tok[1])
        rows.append([int(x) for x in tok[2:22]])
        neff.append(float(tok[22]))
    with open(os.path.join(HERE, "family_pssm.json"), "w") as f:
        json.dump({"source": "demo/family.pssm", "letters": "".join(letters), "query": "".join(qres),
                   "pssm": rows, "neff_2dp": neff}, f)
    shutil.copyfile(os.path.join(ref, "tests", "data", "v1_fixture.fa"), os.path.join(HERE, "v1_fixture.fa"))
    with open(os.path.join(HERE, "v1_fixture_k2_v03.json"), "w") as f:
        json.dump({"source": "tests/data/v1_fixture_k2.v03.m8",
                   "search": "search v1_fixture.fa against itself, --k 2 --mask 0 --evalue 10 --ungapped-xdrop 30 "
                             "--kmer-score 22 --max-kmers 512 --min-diag-score 33",
                   "gaps": [11, 1], "comp_bias": True, "lambda": 0.3649, "k": 0.1076,
                   "hits": parse_m8(os.path.join(ref, "tests", "data", "v1_fixture_k2.v03.m8"))}, f, indent=0)
    print("wrote family.a3m, family_pssm.json, v1_fixture.fa, v1_fixture_k2_v03.json")


if __name__ == "__main__":
    main()
