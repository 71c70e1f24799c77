"""Generate the committed golden fixtures from the IMPACT reference sources (read as text).

Run once in a checkout that has the reference tree:

    python tests/golden/make_golden.py /path/to/GPU-IMPACT-CT

It writes
  fd_exact_table.json    -- every (n_coeff, deltaX, abl) row of the exact equidistant
                            finite-difference weights hard-coded in diff_coeffs_exact
                            (src/mod_coeffs.f90:598-751), as integer numerators and the
                            common denominator;
  stability_limit.json   -- the 41 RK3 stability limits of src/mod_vars.f90:785-795.

The tests compare the oracle's and the library's coefficient generators against these
known answers; nothing at test time reads the reference tree.
"""
import json
import os
import re
import sys


def parse_fd_table(text):
    start = text.index("SUBROUTINE diff_coeffs_exact")
    end = text.index("END SUBROUTINE diff_coeffs_exact")
    body = text[start:end]
    rows = []
    n_cur = None
    for line in body.splitlines():
        line = line.split("!")[0]
        m = re.search(r"IF\s*\(n_coeff\s*==\s*(\d+)\)\s*THEN", line)
        if m:
            n_cur = int(m.group(1))
            continue
        m = re.search(r"IF\s*\(deltaX\s*==\s*([-+]?\d+\.\d*)\s*\.AND\.\s*abl\s*==\s*(\d+)\)\s*"
                      r"cc\(1:n_coeff\)\s*=\s*\(/(.*)/\)\s*/\s*([\d.]+)", line)
        if m and n_cur is not None:
            nums = [float(x) for x in m.group(3).split(",")]
            rows.append({"n": n_cur, "deltaX": float(m.group(1)), "abl": int(m.group(2)),
                         "num": nums, "den": float(m.group(4))})
    return rows


def parse_stability(text):
    start = text.index("stabilitylimit(0:40)")
    seg = text[start:text.index("/)", start)]
    vals = re.findall(r"(\d+\.\d+)", seg)
    return [float(v) for v in vals]


def main(root):
    src = os.path.join(root, "src")
    with open(os.path.join(src, "mod_coeffs.f90"), encoding="latin-1") as f:
        fd = parse_fd_table(f.read())
    with open(os.path.join(src, "mod_vars.f90"), encoding="latin-1") as f:
        stab = parse_stability(f.read())
    assert len(stab) == 41, len(stab)
    assert len(fd) > 100, len(fd)
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "fd_exact_table.json"), "w") as f:
        json.dump({"source": "src/mod_coeffs.f90:598-751 (diff_coeffs_exact)", "rows": fd}, f, indent=0)
    with open(os.path.join(here, "stability_limit.json"), "w") as f:
        json.dump({"source": "src/mod_vars.f90:785-795 (stabilitylimit)", "values": stab}, f, indent=0)
    print(f"wrote {len(fd)} FD rows and {len(stab)} stability limits")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IMPACT_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_golden.py path/to/GPU-IMPACT-CT (or set IMPACT_REFERENCE_ROOT)")
    main(root)
