"""Generate tests/golden/ref_loader.json: the CSR the reference's own loader
builds for each loader edge case of tests/test_host.py (CASES).

The loader is oracle/_ref/ref_load (`make -C oracle ref`): the reference's
unmodified file_reader (util.cpp:19-52) and Graph(1, path) CSR build
(graph.cpp:18-61), compiled from its sources; `ref_load --csr` prints V, E
and the out- and in-CSR it built.  Runs on CPU, wherever the reference
checkout is present:

    python tests/golden/make_ref_loader.py

Only cases inside the reference's defined behaviour are recorded (ids in
range, parseable numbers); the inputs on which it reads out of bounds are
rejected by this repository's loader instead (tests/test_host.py
test_loader_errors).
"""
import json
import os
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF_LOAD = os.path.join(ROOT, "oracle", "_ref", "ref_load")
OUT = os.path.join(ROOT, "tests", "golden", "ref_loader.json")


def parse_csr(text: str):
    """`ref_load --csr` output of one file -> dict."""
    lines = text.splitlines()
    v, e = map(int, lines[0].split())
    rows = [[int(x) for x in ln.split()] for ln in lines[1:5]]
    return {"V": v, "E": e, "out_off": rows[0], "out_adj": rows[1], "in_off": rows[2], "in_adj": rows[3]}


def run_ref_load(path: str):
    out = subprocess.run([REF_LOAD, "--csr", path], capture_output=True, text=True, check=True).stdout
    return parse_csr(out)


def main() -> int:
    sys.path.insert(0, ROOT)
    from tests.test_host import CASES
    if not os.path.exists(REF_LOAD):
        print(f"missing {REF_LOAD}: run make -C oracle ref", file=sys.stderr)
        return 1
    res = {}
    with tempfile.TemporaryDirectory(dir=os.path.dirname(OUT)) as d:
        for name, text in sorted(CASES.items()):
            p = os.path.join(d, name + ".txt")
            with open(p, "w", newline="") as f:
                f.write(text)
            res[name] = run_ref_load(p)
    with open(OUT, "w") as f:  # one case per line
        f.write("{\n" + ",\n".join(f" {json.dumps(k)}: {json.dumps(res[k], sort_keys=True)}"
                                     for k in sorted(res)) + "\n}\n")
    print(f"wrote {len(res)} cases to {OUT}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
