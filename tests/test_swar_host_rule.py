"""The routing rule the library's host code uses for field-parallel sums (`swar_sum_fits_slab` and
`swar_sum_fits_w` in amethyst_b200/csrc/amx_swar.cuh), evaluated by a small host program built
with nvcc (no GPU needed), against the lane model of tests/test_swar_cpu.py: the widths whose
two-field lanes hold a run's sums at the policy's run length, and at the 8 slabs per thread of
the wide count-and-sum variant."""
import os
import subprocess

from tests.test_swar_cpu import sum_fits

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include "amx_swar.cuh"
#include <cstdio>
int main()
{
    for (int b = 1; b <= 32; b++)
        std::printf("%d %d %d\n", b, amx::swar_sum_fits_slab(b) ? 1 : 0, amx::swar_sum_fits_w(b, 8) ? 1 : 0);
    return 0;
}
"""


def test_host_rule_matches_the_lane_model(tmp_path):
    src = tmp_path / "rule.cu"
    exe = tmp_path / "rule"
    src.write_text(PROGRAM)
    cmd = ["nvcc", "-std=c++17", "-O1", "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "amethyst_b200", "csrc"),
           str(src), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    rows = [tuple(int(x) for x in line.split()) for line in out if line.strip()]
    assert [b for b, _, _ in rows] == list(range(1, 33))
    for b, slab, wide in rows:
        e = 64 // b
        spt = 1 if e >= 64 else min(8, 64 // e)
        assert slab == int(sum_fits(b, spt)), b
        assert wide == int(sum_fits(b, 8)), b
    # the wide variant (1-4 bits, 8 slabs per thread) sums in lanes at 4 bits only
    assert [wide for b, _, wide in rows[:4]] == [0, 0, 0, 1]
