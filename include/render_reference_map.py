"""Render aq_reference_map.json (every C entry point of aq.h and the
reference interface it replaces) as the Markdown table of the integration
notes.

    python include/render_reference_map.py            # print the table
    python include/render_reference_map.py NOTES.md    # replace the table in NOTES.md

The table in NOTES.md is the block of lines that starts with the
"| Entry point | Replaces" header row.
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = "| Entry point | Replaces (path in the reference) |"


def rows():
    with open(os.path.join(HERE, "aq_reference_map.json")) as f:
        return json.load(f)["rows"]


def table():
    out = [HEADER, "|---|---|"]
    for r in rows():
        names = r["entry_points"]
        sep = " / " if len(names) <= 4 else ", "
        out.append("| %s | %s |" % (sep.join("`%s`" % n for n in names), r["replaces"]))
    return "\n".join(out)


def replace_in(path):
    with open(path) as f:
        lines = f.read().split("\n")
    a = next(i for i, ln in enumerate(lines) if ln.startswith("| Entry point | Replaces"))
    b = a
    while b < len(lines) and lines[b].startswith("|"):
        b += 1
    lines[a:b] = table().split("\n")
    with open(path, "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    if len(sys.argv) > 1:
        replace_in(sys.argv[1])
    else:
        print(table())
