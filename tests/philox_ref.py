"""Test-side Philox4x32-10 (Salmon et al., SC'11), xoshiro128** and the shuffle the device runs.

Used to predict, configuration by configuration, what the random mode evaluates: configuration g of a job
is the shuffle of the packed arrangement whose words come from a xoshiro128** generator seeded with the
Philox block of counter (0, iteration, g_lo, g_hi << 8 | part) and key (seed_lo, seed_hi), bounded like
core/shuffle.h:28-32 of the reference: p = (x * i) >> 32. Each window in turn takes a Fisher-Yates pass,
or, when it holds exactly two species and the binary_floyd option is on (the default), Floyd's sampling of
the sites of its rarer species (ties: the higher species index) over the window filled with the other one.
"""
M0, M1 = 0xD2511F53, 0xCD9E8D57
W0, W1 = 0x9E3779B9, 0xBB67AE85
MASK = 0xFFFFFFFF

# Published known-answer vectors of philox4x32-10 (Random123 distribution).
KATS = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((MASK, MASK, MASK, MASK), (MASK, MASK), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


def philox4x32_10(ctr, key):
    c0, c1, c2, c3 = ctr
    k0, k1 = key
    for _ in range(10):
        p0 = M0 * c0
        p1 = M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & MASK, p1 & MASK, ((p0 >> 32) ^ c3 ^ k1) & MASK, p0 & MASK
        k0 = (k0 + W0) & MASK
        k1 = (k1 + W1) & MASK
    return c0, c1, c2, c3


def rotl32(x, k):
    return ((x << k) | (x >> (32 - k))) & MASK


class Xoshiro128ss:
    """xoshiro128** (Blackman and Vigna, ACM TOMS 2021): 128-bit state, 32-bit outputs."""

    def __init__(self, s):
        self.s = list(s)
        if not any(self.s):
            self.s[0] = 1

    def next(self):
        s0, s1, s2, s3 = self.s
        r = (rotl32((s1 * 5) & MASK, 7) * 9) & MASK
        t = (s1 << 9) & MASK
        s2 ^= s0
        s3 ^= s1
        s1 ^= s2
        s0 ^= s3
        s2 ^= t
        s3 = rotl32(s3, 11)
        self.s = [s0, s1, s2, s3]
        return r


def floyd_choice(window):
    """(m, rare, other) of a window of exactly two species, else None: rare is the species with fewer
    sites (ties: the higher index) and m its site count."""
    values = sorted(set(window))
    if len(values) != 2:
        return None
    a, b = values
    na, nb = window.count(a), window.count(b)
    rare, other = (b, a) if nb <= na else (a, b)
    return min(na, nb), rare, other


def shuffle(species, windows, seed, chain, iteration, part=0, floyd=True):
    """One shuffle of every window, in place on a list: the words come from a xoshiro128** generator
    whose state is the Philox4x32-10 block of counter (0, iteration, chain_lo, chain_hi << 8 | part) and
    key (seed_lo, seed_hi). ``species`` must be the packed arrangement (the rule that picks Floyd's
    sampling reads each window's species)."""
    k = (seed & MASK, (seed >> 32) & MASK)
    c_lo = chain & MASK
    c_hi = (((chain >> 32) << 8) | part) & MASK
    gen = Xoshiro128ss(philox4x32_10((0, iteration & MASK, c_lo, c_hi), k))
    for lo, hi in windows:
        n = hi - lo
        choice = floyd_choice(species[lo:hi]) if floyd else None
        if choice is not None:
            m, rare, other = choice
            species[lo:hi] = [other] * n
            for j in range(n - m, n):
                t = (gen.next() * (j + 1)) >> 32
                species[lo + (j if species[lo + t] == rare else t)] = rare
            continue
        for i in range(n, 1, -1):
            p = (gen.next() * i) >> 32
            a, b = lo + i - 1, lo + p
            species[a], species[b] = species[b], species[a]
    return species
