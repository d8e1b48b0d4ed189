"""Synthetic inputs for the tests and the benchmark: not part of the product.

* workloads: seeded generators with the shapes of the five benchmark
  configurations (SplitMix64 streams, BLOSUM62 background residues, planted
  homologs, family MSAs);
* profile: PSSM rows from MSAs through synth/libsynth.so (a host restatement of
  the reference's src/profile.rs, pinned by its demo/family.pssm).

Nothing here loads libsabertooth_b200.so, so a process that only generates
inputs (the CPU reference arm of bench.py) maps no product code.
"""
