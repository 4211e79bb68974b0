"""The random stream without a GPU: the test-side Philox4x32-10 against the published Random123
known-answer vectors, and the library's host build of philox.cuh (Philox4x32-10 and the xoshiro128**
words that feed every random shuffle) against the test-side implementation that the GPU tests use to
predict each evaluated configuration."""
import os
import subprocess

import philox_ref

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <cstdio>
#include "philox.cuh"
using namespace sqsg;
int main() {
  unsigned c[4], k[2], it, clo, chi, k0, k1;
  char what[8];
  while (std::scanf("%7s", what) == 1) {
    if (what[0] == 'p') {
      std::scanf("%u %u %u %u %u %u", &c[0], &c[1], &c[2], &c[3], &k[0], &k[1]);
      philox_ctr r = philox4x32_10(philox_ctr{c[0], c[1], c[2], c[3]}, k[0], k[1]);
      std::printf("%u %u %u %u\n", r.x, r.y, r.z, r.w);
    } else {
      std::scanf("%u %u %u %u %u", &it, &clo, &chi, &k0, &k1);
      xoshiro128ss g = shuffle_words(it, clo, chi, k0, k1);
      for (int n = 0; n < 16; ++n) std::printf("%u%c", g.next(), n == 15 ? '\n' : ' ');
    }
  }
  return 0;
}
"""


def test_philox_known_answers():
    for ctr, key, want in philox_ref.KATS:
        assert philox_ref.philox4x32_10(ctr, key) == want


def test_host_build_matches_test_side_stream(tmp_path):
    src = tmp_path / "rng.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "rng"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "sqsgenerator_b200", "csrc"), str(src),
                    "-o", str(exe)], check=True)
    M = philox_ref.MASK
    lines, want = [], []
    for ctr, key, _ in philox_ref.KATS:
        lines.append("p %d %d %d %d %d %d" % (*ctr, *key))
        want.append(" ".join(str(x) for x in philox_ref.philox4x32_10(ctr, key)))
    for it, chain, part, seed in ((0, 0, 0, 0), (0, 1, 0, 42), (0, 2_097_152, 1, 0x1234_5678_9ABC),
                                  (3, (7 << 32) + 5, 2, M)):
        clo, chi = chain & M, (((chain >> 32) << 8) | part) & M
        k0, k1 = seed & M, (seed >> 32) & M
        lines.append("w %d %d %d %d %d" % (it, clo, chi, k0, k1))
        gen = philox_ref.Xoshiro128ss(philox_ref.philox4x32_10((0, it, clo, chi), (k0, k1)))
        want.append(" ".join(str(gen.next()) for _ in range(16)))
    out = subprocess.run([str(exe)], input="\n".join(lines) + "\n", capture_output=True, text=True, check=True)
    assert out.stdout.split("\n")[: len(want)] == want


def test_shuffle_is_a_permutation_of_each_window():
    species = [0] * 10 + [1] * 12 + [2] * 10
    windows = [(0, 22), (22, 32)]
    for g in range(50):
        conf = philox_ref.shuffle(list(species), windows, 99, g, 0)
        assert sorted(conf[:22]) == sorted(species[:22]) and sorted(conf[22:]) == sorted(species[22:])


def test_floyd_windows_take_every_arrangement_equally_often():
    """Floyd's sampling on a two-species window (6 sites, 2 of the rarer species: 15 arrangements) and
    Fisher-Yates on the same window give each arrangement with probability 1/15: chi-square of 15,000
    seeded configurations against uniform, far below the 0.1 % point of 14 degrees of freedom (36.1)."""
    species = [1, 1, 0, 0, 0, 0]
    assert philox_ref.floyd_choice(species) == (2, 1, 0)
    assert philox_ref.floyd_choice([0, 0, 1, 1]) == (2, 1, 0)  # ties: the higher species index
    assert philox_ref.floyd_choice([0, 1, 2]) is None
    for floyd in (True, False):
        seen = {}
        for g in range(15_000):
            conf = tuple(philox_ref.shuffle(list(species), [(0, 6)], 7, g, 0, floyd=floyd))
            assert sorted(conf) == sorted(species)
            seen[conf] = seen.get(conf, 0) + 1
        assert len(seen) == 15
        chi2 = sum((c - 1000) ** 2 / 1000 for c in seen.values())
        assert chi2 < 36.1, (floyd, chi2)


def test_floyd_window_draws_m_words():
    """A two-species window takes one word per site of its rarer species: the next window's draws start
    m words into the stream (here m = 3 of 10 sites, then a three-species window)."""
    species = [0] * 7 + [1] * 3 + [0, 1, 2, 2]
    windows = [(0, 10), (10, 14)]
    k, it, g = 5, 0, 11
    got = philox_ref.shuffle(list(species), windows, k, g, it)
    gen = philox_ref.Xoshiro128ss(philox_ref.philox4x32_10((0, it, g, 0), (k, 0)))
    want = [0] * 10
    for j in range(7, 10):
        t = (gen.next() * (j + 1)) >> 32
        want[j if want[t] == 1 else t] = 1
    tail = species[10:]
    for i in range(4, 1, -1):
        p = (gen.next() * i) >> 32
        tail[i - 1], tail[p] = tail[p], tail[i - 1]
    assert got == want + tail
