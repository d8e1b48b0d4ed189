"""The reference tests' xorshift64 generator (src/simd.rs:1072-1086) and
SplitMix64 (src/evalue.rs:54-75), so parity cases are drawn the way the
reference's own tests draw theirs."""

MASK = (1 << 64) - 1


class XorShift:
    def __init__(self, seed):
        self.s = seed & MASK

    def next(self):
        x = self.s
        x ^= (x << 13) & MASK
        x ^= x >> 7
        x ^= (x << 17) & MASK
        self.s = x
        return x

    def range(self, n):
        return self.next() % n

    below = range


class SplitMix64:
    def __init__(self, seed):
        self.s = seed & MASK

    def next_u64(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def below(self, n):
        return self.next_u64() % n

    def next_f64(self):
        # (next_u64() >> 11) / 2^53, exact in binary64 (src/evalue.rs:70-72)
        return (self.next_u64() >> 11) / float(1 << 53)


def rand_seq(rng, length, alpha):
    return [rng.range(alpha) for _ in range(length)]
