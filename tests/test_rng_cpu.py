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
