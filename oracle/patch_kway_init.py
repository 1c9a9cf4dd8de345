"""Build step of oracle/Makefile (test infrastructure only): a copy of the reference's
sources/main.cu whose k-way initial partition runs the reference's own GPU routine
`initial_partitioning` (sources/init_part.cu:186-727) instead of the external Mt-KaHyPar binary
(`initial_partitioning_kahypar`, sources/init_part.cu:733-953).

The reference keeps that GPU routine dormant: both k-way base cases in main.cu (the node-count
threshold at :359-372 and the shrink-ratio case at :449-462) hold its call in a comment, followed
by the live Mt-KaHyPar call. This script swaps the two in each place and writes the result to the
given output path (under oracle/_ref/, git-ignored). Mt-KaHyPar is absent on this machine, so this
"reference-family" build is the only way to run the reference's k-way path here; its numbers are
labelled as such, never as the reference's Mt-KaHyPar result.

    python3 patch_kway_init.py <reference main.cu> <output .cu>
"""
import re
import sys

PATTERN = re.compile(
    r"/\*(auto \[d_init_partitions, d_init_partitions_sizes\] = initial_partitioning\((?:.|\n)*?\);)\*/"
    r"(\s*)"
    r"(auto \[d_init_partitions, d_init_partitions_sizes\] = initial_partitioning_kahypar\((?:.|\n)*?\);)")


def main() -> int:
    src, dst = sys.argv[1], sys.argv[2]
    with open(src) as f:
        text = f.read()
    out, count = PATTERN.subn(lambda m: m.group(1) + m.group(2) + "/*" + m.group(3) + "*/", text)
    if count != 2:
        print(f"patch_kway_init: expected 2 k-way base cases in {src}, found {count}", file=sys.stderr)
        return 1
    with open(dst, "w") as f:
        f.write(out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
