"""Regenerate blosum62.json from the reference's blosum62.out.

Restates SubstitutionMatrix::from_out_str (reference src/matrix.rs:56-175) with
bit factor 2.0 and bias -0.2 (src/matrix.rs:50-52): parse the half-bit
log-odds file, rescale the background when X is not positive (ANY_BACK =
1e-5), rebuild the joint probabilities P(a,b) = exp(lambda*S_ab) * pa * pb,
the pseudocount matrix R[a][b] = P(a,b)/pb as f32, and the integer matrix
round(bit_factor * log2(P/(pa*pb)) + bias) rounded half away from zero and
clamped to int8.  math.exp / math.log2 call the platform libm, as the
reference's f64::exp / f64::log2 do.

Run where the reference tree is present:
    python sabertooth_b200/data/make_blosum62.py /path/to/reference/src/data/blosum62.out
"""
import json
import math
import os
import sys

import numpy as np

LETTERS = "ACDEFGHIKLMNPQRSTVWYX"  # src/alphabet.rs:8-10


def aa2num(ch):
    u = ch.upper()
    return LETTERS.index(u) if u in LETTERS else 20


def build(text, bit_factor=2.0, bias=-0.2):
    A = 21
    raw = [[0.0] * A for _ in range(A)]
    p_back = [0.0] * A
    lam = None
    cols = None
    for line in text.splitlines():
        t = line.rstrip()
        if not t:
            continue
        bg = "# Background (precomputed optional):"
        lm = "# Lambda     (precomputed optional):"
        if t.startswith(bg):
            for i, tok in enumerate(t[len(bg):].split()):
                if i < A:
                    p_back[i] = float(tok)
            continue
        if t.startswith(lm):
            lam = float(t[len(lm):].strip())
            continue
        if t.startswith("#"):
            continue
        toks = t.split()
        if cols is None:
            if all(len(x) == 1 and x.isalpha() for x in toks):
                cols = [aa2num(x) for x in toks]
            continue
        if not toks[0][0].isalpha():
            continue
        row = aa2num(toks[0][0])
        for j, tok in enumerate(toks[1:]):
            if j < len(cols):
                raw[row][cols[j]] = float(tok)
    assert lam is not None
    x = 20
    x_pos = any(raw[x][j] > 0.0 or raw[j][x] > 0.0 for j in range(A))
    if not x_pos:
        p_back[x] = 1e-5
        for i in range(20):
            p_back[i] *= 1.0 - p_back[x]
    prob = [[math.exp(lam * raw[i][j]) * p_back[i] * p_back[j] for j in range(A)] for i in range(A)]
    r = [[float(np.float32(prob[a][b] / p_back[b])) for b in range(20)] for a in range(20)]
    score = [[0] * A for _ in range(A)]
    for i in range(A):
        for j in range(A):
            s = prob[i][j] / (p_back[i] * p_back[j])
            val = bit_factor * math.log2(s) + bias
            rounded = val - 0.5 if val < 0.0 else val + 0.5
            rounded = min(max(rounded, -128.0), 127.0)
            score[i][j] = int(rounded)  # truncation toward zero, as `as i8`
    return {"name": "blosum62", "letters": LETTERS, "bit_factor": bit_factor, "bias": bias, "lambda": lam,
            "p_back": p_back, "prob": prob, "r": r, "score": score}


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_blosum62.py /path/to/reference/src/data/blosum62.out")
    src = sys.argv[1]
    with open(src) as f:
        data = build(f.read())
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "blosum62.json")
    with open(out, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()
