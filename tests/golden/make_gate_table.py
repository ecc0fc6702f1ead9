"""Extracts the node-gate blocks of the reference's periodic 3-point CUDA
kernels from their source text: XXX3iso_BPC / XXY3iso_BPC
(cuda/kernels/3isoBPC_k.cuh) and XXX3ani_BPC / XXY3ani_BPC
(cuda/kernels/3aniBPC_k.cuh).  Each kernel runs its point loop from 64
`count123*` calls, each nested in `if` conditions on the node distances and
edge flags; this script records, per call in source order, the image flags
it passes and its gate (the flags it requires and its node-distance tests),
checks that all four kernels hold the same 64 blocks, and writes them to
gate_table.json in the form of node_gates.cuh's kGateBlocks:

    [f2, f3, a2, a3, [[pair, k, [axes...]], ...]]

f2 / f3 / a2 / a3 are bit masks (bit 0 x, 1 y, 2 z); pair 0, 1, 2 = nodes
12, 23, 31; a test reads dd_pair + k*L^2 - 2*(sum of |dn_pair| over axes)*L
<= d_max_node, k = 0 without axes meaning dd_pair <= d_max_node.

    python tests/golden/make_gate_table.py [REFERENCE_ROOT]

The reference root comes from the argument or, failing that, the
PCF_REFERENCE_ROOT environment variable."""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
AXIS = {"x": 0, "y": 1, "z": 2}
PAIR = {"12": 0, "23": 1, "31": 2}


def _kernel_body(lines, name):
    """Line range of the __global__ function `name`."""
    start = next(i for i, ln in enumerate(lines) if "__global__" in ln and f" {name}(" in ln)
    depth, seen = 0, False
    for i in range(start, len(lines)):
        depth += lines[i].count("{") - lines[i].count("}")
        seen = seen or "{" in lines[i]
        if seen and depth == 0:
            return start, i + 1
    raise ValueError(name)


def _blocks(lines, lo, hi):
    stack, depth, assign, out = [], 0, {}, []
    for ln in lines[lo:hi]:
        s = ln.strip()
        m = re.match(r"if \((.*)\)\s*\{$", s)
        if m:
            stack.append((depth, m.group(1)))
        m = re.match(r"(f_dd_nod\d\d) = (.*);", s)
        if m:
            assign[m.group(1)] = m.group(2)
        if re.search(r"\bcount123\w*\(", s):
            flags = re.findall(r"\b(true|false)\b", s)[-6:]
            f = [1 if v == "true" else 0 for v in flags]
            conds = []
            for _, c in stack:
                for k, v in assign.items():
                    c = c.replace(k, "[" + v + "]")
                conds.append(c)
            out.append((f, " && ".join(conds)))
        depth += s.count("{") - s.count("}")
        while stack and stack[-1][0] >= depth:
            stack.pop()
    return out


def _parse(flags, cond):
    f2 = flags[0] | flags[1] << 1 | flags[2] << 2
    f3 = flags[3] | flags[4] << 1 | flags[5] << 2
    a2 = a3 = 0
    tests = []
    for t in (t.strip() for t in re.split(r"&&(?![^\[]*\])", cond)):
        if re.match(r"idx\d<", t):
            continue
        m = re.fullmatch(r"f([xyz])_([23])", t)
        if m:
            if m.group(2) == "2":
                a2 |= 1 << AXIS[m.group(1)]
            else:
                a3 |= 1 << AXIS[m.group(1)]
            continue
        if re.fullmatch(r"\(f[xyz]_[23] \|\| f[xyz]_[23] \|\| f[xyz]_[23]\)", t):
            continue  # implied by the flags each block requires
        m = re.fullmatch(r"dd_nod(\d\d) <= d_max_node", t)
        if m:
            tests.append([PAIR[m.group(1)], 0, []])
            continue
        m = re.fullmatch(r"\[dd_nod(\d\d) \+ (?:(\d)\*)?size_box2 - 2\*\(?([^)]*?)\)?\*size_box\] "
                         r"<= d_max_node", t)
        if m:
            toks = re.findall(r"d([xyz])n(\d\d)", m.group(3))
            assert all(p == m.group(1) for _, p in toks), t
            tests.append([PAIR[m.group(1)], int(m.group(2) or 1), [AXIS[a] for a, _ in toks]])
            continue
        raise ValueError("unparsed condition: " + t)
    return [f2, f3, a2, a3, tests]


def extract(ref):
    tables = []
    for fname, kernels in (("3isoBPC_k.cuh", ("XXX3iso_BPC", "XXY3iso_BPC")),
                           ("3aniBPC_k.cuh", ("XXX3ani_BPC", "XXY3ani_BPC"))):
        lines = open(os.path.join(ref, "cuda", "kernels", fname)).read().split("\n")
        for k in kernels:
            lo, hi = _kernel_body(lines, k)
            blocks = [_parse(f, c) for f, c in _blocks(lines, lo, hi)]
            assert len(blocks) == 64, (k, len(blocks))
            tables.append(blocks)
    assert all(t == tables[0] for t in tables), "the four kernels' blocks differ"
    return tables[0]


def main():
    ref = next((a for a in sys.argv[1:]), os.environ.get("PCF_REFERENCE_ROOT"))
    if not ref:
        sys.exit("usage: make_gate_table.py REFERENCE_ROOT (or set PCF_REFERENCE_ROOT)")
    table = extract(ref)
    with open(os.path.join(HERE, "gate_table.json"), "w") as f:
        json.dump(table, f)
    print(len(table), "blocks")


if __name__ == "__main__":
    main()
