"""Extract the known-answer vectors of HybridSmoothers.jl's own test suite into
tests/golden/reference_kats.json.

The reference is Julia and cannot run here, so its golden vectors are taken
from its test sources, read as text.  Each entry records the file and line it
came from.  Run once, where the reference checkout is available:

    python tests/golden/make_reference_kats.py /path/to/HybridSmoothers.jl

The JSON it writes is committed; tests never read the reference tree.
"""
import json
import os
import re
import sys

# (key, file, regex on a single line, group holding the Julia vector literal)
PATTERNS = [
    ("y_exp_fwd", "test/test_preconditioners.jl", r"y_exp_fwd = (\[.*\])"),
    ("y_exp_bwd", "test/test_preconditioners.jl", r"y_exp_bwd = (\[.*\])"),
    ("y_exp_sym", "test/test_preconditioners.jl", r"y_exp_sym = (\[.*\])"),
    ("D_Dl1_exp", "test/test_preconditioners.jl", r"^\s+D_Dl1_exp = Float64\.\((\[.*\])\)\s+#.*2 >= 1\.5\*1"),
    ("SLbuffer_exp", "test/test_preconditioners.jl", r"^\s+SLbuffer_exp = Float64\.\((\[-1, -1, -1, -1\])"),
    ("SUbuffer_exp", "test/test_preconditioners.jl", r"^\s+SUbuffer_exp = Float64\.\((\[-1, -1, -1, -1\])"),
    ("D_Dl1_eta3", "test/test_preconditioners.jl", r"D_Dl1_exp = Float64\.\((\[2\.0, 2\.5.*\])"),
    ("y2_fwd_exp", "test/test_preconditioners.jl", r"y2_fwd_exp = (\[.*\])"),
    ("y2_bwd_exp", "test/test_preconditioners.jl", r"y2_bwd_exp = (\[[^#]*\])"),
    ("D_Dl1_exp2", "test/test_preconditioners.jl", r"D_Dl1_exp2 = Float64\.\((\[.*\])"),
    ("SLbuffer_exp_ps3", "test/test_preconditioners.jl", r"SLbuffer_exp = Float64\.\((\[-1, 0, .*\])"),
    ("l1_rowsum_poisson5", "test/test_chebyshev.jl", r"_l1_rowsum\(A\) ≈ (\[.*\])"),
    ("gpu_y_exp_fwd", "test/gpu/gpu.jl", r"y_exp_fwd = (\[.*\])"),
    ("gpu_y_exp_bwd", "test/gpu/gpu.jl", r"y_exp_bwd = (\[.*\])"),
    ("gpu_y_exp_sym", "test/gpu/gpu.jl", r"y_exp_sym = (\[.*\])"),
]


def julia_vec(lit):
    body = lit.strip()[1:-1]
    out = []
    for tok in body.split(","):
        tok = tok.strip()
        if not tok:
            continue
        if "/" in tok:
            a, b = tok.split("/")
            out.append(float(a) / float(b))
        else:
            out.append(float(tok))
    return out


def main(ref):
    kats = {}
    for key, rel, rx in PATTERNS:
        lines = open(os.path.join(ref, rel), encoding="utf-8").read().splitlines()
        for no, line in enumerate(lines, 1):
            m = re.search(rx, line)
            if m:
                kats[key] = {"value": julia_vec(m.group(1)), "source": f"{rel}:{no}"}
                break
        else:
            raise SystemExit(f"pattern for {key} not found in {rel}")
    # The a* table in the ChebyshevFirst docstring (src/chebyshev.jl), 3 digits.
    lines = open(os.path.join(ref, "src/chebyshev.jl"), encoding="utf-8").read().splitlines()
    table, src = {}, []
    for no, line in enumerate(lines, 1):
        for k, v in re.findall(r"k=(\d+): (?:a\*≈)?(0\.\d+)", line):
            table[int(k)] = float(v)
            src.append(no)
    kats["astar_table"] = {"value": [table[k] for k in sorted(table)],
                           "source": f"src/chebyshev.jl:{min(src)}-{max(src)}"}
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")
    with open(out, "w") as f:
        json.dump(kats, f, indent=1)
    print(f"wrote {out} ({len(kats)} vectors)")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_reference_kats.py <path of the HybridSmoothers.jl checkout>")
    main(sys.argv[1])
