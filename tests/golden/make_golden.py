"""Regenerate the golden fixtures of this directory from the reference tree.

* family.a3m / family_pssm.json: the reference's demo MSA and the PSSM it
  wrote for it (demo/family.a3m, demo/family.pssm; `sabertooth profile`
  output): pins the PSSM construction that builds PSSM query rows.

Run where the reference tree is present:
    python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
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
    print("wrote family.a3m, family_pssm.json")


if __name__ == "__main__":
    main()
