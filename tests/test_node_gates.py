"""CPU: the reference kernels' node-gate table (PCF_REF_NODE_GATES) is
restated twice, for the GPU (desi_b200/csrc/node_gates.cuh) and in the
oracle (oracle/pcf_oracle.c).  Both copies hold the same 64 blocks, and the
GPU's index by image lists exactly the blocks with those image flags.  (The
blocks themselves are pinned to the reference's kernels by
test_oracle_reference_gates_equal_reference_kernels.)"""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _table(path, name):
    src = open(os.path.join(ROOT, path)).read()
    i = src.index(name)
    body = src[src.index("{", i) + 1:]
    depth, out = 1, []
    for ch in body:
        if ch == "{":
            depth += 1
        elif ch == "}":
            depth -= 1
            if depth == 0:
                break
        out.append(ch)
    return [int(v) for v in re.findall(r"-?\d+", "".join(out))]


def test_gpu_and_oracle_gate_tables_are_the_same():
    gpu = _table("desi_b200/csrc/node_gates.cuh", "kGateBlocks[64]")
    orc = _table("oracle/pcf_oracle.c", "kGates[64]")
    assert len(gpu) == 64 * 19 and gpu == orc


def test_index_by_image_matches_the_blocks():
    blocks = _table("desi_b200/csrc/node_gates.cuh", "kGateBlocks[64]")
    by = _table("desi_b200/csrc/node_gates.cuh", "kGateByImage[64][2]")
    assert len(by) == 128
    for img in range(64):
        want = [b for b in range(64) if blocks[19 * b] | (blocks[19 * b + 1] << 3) == img]
        got = [b for b in by[2 * img:2 * img + 2] if b >= 0]
        assert got == want, img
    # the reference's blocks cover every image pair but (y, xyz) once, and
    # (x, xyz) twice (its block 33 counts with node 2's x image)
    counts = [sum(1 for b in by[2 * i:2 * i + 2] if b >= 0) for i in range(64)]
    assert counts.count(1) == 62 and counts[2 | (7 << 3)] == 0 and counts[1 | (7 << 3)] == 2


def test_gpu_gate_table_is_the_reference_source():
    """kGateBlocks equals the blocks extracted from the reference's kernel
    source (tests/golden/gate_table.json, made by
    tests/golden/make_gate_table.py from 3isoBPC_k.cuh and 3aniBPC_k.cuh,
    whose four kernels hold the same 64 blocks)."""
    import json
    ref = json.load(open(os.path.join(ROOT, "tests", "golden", "gate_table.json")))
    flat = []
    for f2, f3, a2, a3, tests in ref:
        flat += [f2, f3, a2, a3]
        for pair, k, axes in tests:
            flat += [pair, k] + axes + [-1] * (3 - len(axes))
    assert _table("desi_b200/csrc/node_gates.cuh", "kGateBlocks[64]") == flat
