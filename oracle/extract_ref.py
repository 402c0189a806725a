"""Build step for the reference harness (oracle/_ref): writes a translation unit
that #includes line ranges of the reference's gkc_cuda.cu, so its device
kernels compile as host C++ behind oracle/ref_shim.h; with "stats" as the
third argument, the partition-size report calVarStdev of experiment.cpp
instead.

The reference file cannot be compiled whole by a host compiler because its
host driver uses the <<<...>>> launch syntax, so only the ranges holding the
constant tables and the kernels are taken.  Each range is anchored on a line
whose text is checked, so a different reference revision fails loudly rather
than compiling something else.  Output goes to oracle/_ref/ only.

Usage: python extract_ref.py <reference_root> <out_file> [stats]
"""
import sys

# (first line, last line, anchor text expected on the first line)
RANGES = [
    (1, 8, "#define _in_"),                     # FILTER_KERNEL selection (:6)
    (25, 93, "d_basemap[256]"),                 # code tables
    (146, 339, "struct T_d_data"),              # HPC, filters, minimizer, GenSKM, MoveOffset
    (350, 365, "CalcSKMPartSize_instream"),     # per-bin superkmer bases
]
# experiment.cpp: calVarStdev, the avg / max / min / var / std / cv report
STATS_RANGE = (18, 37, "void calVarStdev")
FILTER_LINE = 6  # "#define FILTER_KERNEL new_filter2"
ANCHORS = {
    FILTER_LINE: "#define FILTER_KERNEL",
    164: "GPU_HPCEncoding",
    234: "GPU_GenMinimizer",
    298: "GPU_GenSKM",
    331: "MoveOffset",
}


def extract_stats(ref_root, out):
    path = f"{ref_root}/experiment.cpp"
    lines = open(path, encoding="utf-8", errors="replace").read().split("\n")
    a, b, text = STATS_RANGE
    if text not in lines[a - 1]:
        raise SystemExit(f"{path}:{a}: expected '{text}', found '{lines[a - 1]}'")
    with open(out, "w") as f:
        f.write("// generated by oracle/extract_ref.py -- not source\n")
        f.write(f'#line {a} "{path}"\n')
        for ln in range(a, b + 1):
            f.write(lines[ln - 1] + "\n")


def main():
    ref_root, out = sys.argv[1], sys.argv[2]
    if len(sys.argv) > 3 and sys.argv[3] == "stats":
        return extract_stats(ref_root, out)
    path = f"{ref_root}/gkc_cuda.cu"
    lines = open(path, encoding="utf-8", errors="replace").read().split("\n")
    for ln, text in list(ANCHORS.items()) + [(a, t) for a, _, t in RANGES]:
        if text not in lines[ln - 1]:
            raise SystemExit(f"{path}:{ln}: expected '{text}', found '{lines[ln - 1]}'")
    with open(out, "w") as f:
        f.write("// generated by oracle/extract_ref.py -- not source\n")
        for a, b, _ in RANGES:
            f.write(f'#line {a} "{path}"\n')
            for ln in range(a, b + 1):
                text = lines[ln - 1]
                if ln == FILTER_LINE:
                    # the filter stays selectable: -DFILTER_KERNEL=<variant>
                    f.write("#ifndef FILTER_KERNEL\n" + text + "\n#endif\n")
                    f.write(f'#line {ln + 1} "{path}"\n')
                else:
                    f.write(text + "\n")


if __name__ == "__main__":
    main()
