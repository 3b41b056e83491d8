"""Graph format converters (the reference's data tooling, restated).

* ``snap_to_cuts``: a SNAP edge list (``#`` comment lines, ``s<TAB>t``) to the
  cuTS text format, whose first line is max vertex id + 1 -- the same rule as
  the reference's data_set/data/cuts_graph_converter.py:13-23.
* ``cuts_to_gsi``: a cuTS query file to GSI's input format, every vertex and
  edge labelled 1 -- as data_set/query/convert_ours_to_gsi.py:4-20.

    python -m cuts_b200.convert snap2cuts in.txt out.g
    python -m cuts_b200.convert cuts2gsi in.g out.g
"""
import sys


def snap_to_cuts(src: str, dst: str) -> int:
    edges = []
    max_id = -1
    with open(src) as f:
        for line in f:
            if "#" in line:
                continue
            parts = line.split("\t")
            if len(parts) < 2:
                continue
            s, t = int(parts[0]), int(parts[1])
            max_id = max(max_id, s, t)
            edges.append(line if line.endswith("\n") else line + "\n")
    with open(dst, "w") as f:
        f.write(f"{max_id + 1}\n")
        f.writelines(edges)
    return max_id + 1


def cuts_to_gsi(src: str, dst: str) -> None:
    with open(src) as f:
        lines = f.readlines()
    n = int(lines[0])
    out = ["t # 0\n", f"{n} {len(lines) - 1} 1 1\n"]
    out += [f"v {i} 1\n" for i in range(n)]
    for line in lines[1:]:
        parts = line.split("\t")
        out.append(f"e {int(parts[0])} {int(parts[1])} 1\n")
    out.append("t # -1\n")
    with open(dst, "w") as f:
        f.writelines(out)


def main(argv=None):
    argv = argv if argv is not None else sys.argv[1:]
    if len(argv) != 3 or argv[0] not in ("snap2cuts", "cuts2gsi"):
        print(__doc__)
        return 2
    (snap_to_cuts if argv[0] == "snap2cuts" else cuts_to_gsi)(argv[1], argv[2])
    return 0


if __name__ == "__main__":
    sys.exit(main())
