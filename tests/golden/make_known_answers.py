"""Writes tests/golden/known_answers.json: the known answers of the
reference's own unit tests (javagg/rmetis, Rust), transcribed from their
source with file:line. The reference cannot be built or run here (no Rust
toolchain), so these literal tables are the fixture; tests/test_golden.py
checks the oracle (CPU) and the GPU library against them.

    python tests/golden/make_known_answers.py
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))

# Graphs built by the reference's tests.
GRAPHS = {
    # cycle 0-1-2-3-0 (src/graph/mod.rs tests, src/graph/validate.rs:148-149,
    # src/refine/greedy.rs:225-227)
    "cycle4": {"xadj": [0, 2, 4, 6, 8], "adjncy": [1, 3, 0, 2, 1, 3, 0, 2]},
    # path 0-1-2-3 (src/graph/mod.rs:500-505, src/coarsen/rm.rs:52-54)
    "path4": {"xadj": [0, 1, 3, 5, 6], "adjncy": [1, 0, 2, 1, 3, 2]},
    # star with a heavy edge 0-2 (src/coarsen/shem.rs:86-93)
    "star4_w": {"xadj": [0, 3, 4, 5, 6], "adjncy": [1, 2, 3, 0, 0, 0], "adjwgt": [1, 3, 1, 1, 3, 1]},
    # 2x2 grid (src/initial/grow.rs:112-119)
    "grid4": {"xadj": [0, 2, 4, 6, 8], "adjncy": [1, 2, 0, 3, 0, 3, 1, 2]},
    # 3x3 grid, rebuilt with sorted rows (src/refine/fm_kway.rs:165-206)
    "grid3x3": {"xadj": [0, 2, 5, 7, 10, 14, 17, 19, 22, 24],
                "adjncy": [1, 3, 0, 2, 4, 1, 5, 0, 4, 6, 1, 3, 5, 7, 2, 4, 8, 3, 7, 4, 6, 8, 5, 7]},
}

CASES = [
    {"kind": "edge_cut", "graph": "cycle4", "part": [0, 0, 1, 1], "expect": 2,
     "ref": "src/graph/mod.rs:454-461"},
    {"kind": "partition_weights", "graph": "cycle4", "part": [0, 0, 1, 1], "nparts": 2, "expect": [[2], [2]],
     "ref": "src/graph/mod.rs:463-470"},
    {"kind": "total_weight", "graph": "cycle4", "expect": [4], "ref": "src/graph/mod.rs:472-476"},
    {"kind": "boundary", "graph": "cycle4", "part": [0, 0, 1, 1], "expect": [0, 1, 2, 3],
     "ref": "src/graph/mod.rs:478-485"},
    {"kind": "coarse", "graph": "path4", "matching": [1, 0, 3, 2],
     "expect": {"nvtxs": 2, "nedges": 1, "same": [[0, 1], [2, 3]], "different": [[0, 2]]},
     "ref": "src/graph/mod.rs:498-514"},
    {"kind": "validate", "n": 4, "xadj": [0, 2, 4, 6, 8], "adjncy": [1, 3, 0, 2, 1, 3, 0, 2], "expect": "ok",
     "ref": "src/graph/validate.rs:151-154 valid_square"},
    {"kind": "validate", "n": 4, "xadj": [0, 2, 4], "adjncy": [1, 3, 0, 2, 1, 3, 0, 2], "expect": "reject",
     "ref": "src/graph/validate.rs:156-161 wrong_xadj_len"},
    {"kind": "validate", "n": 4, "xadj": [0, 3, 5, 7, 9], "adjncy": [0, 1, 3, 0, 2, 1, 3, 0, 2], "expect": "reject",
     "ref": "src/graph/validate.rs:163-170 self_loop"},
    {"kind": "validate", "n": 4, "xadj": [0, 1, 1, 0, 0], "adjncy": [1], "expect": "reject",
     "ref": "src/graph/validate.rs:172-180 asymmetric"},
    {"kind": "validate", "n": 4, "xadj": [0, 2, 4, 6, 8], "adjncy": [1, 3, 0, 2, 1, 3, 0, 2], "vwgt": [1, 1, 1],
     "expect": "reject", "ref": "src/graph/validate.rs:182-188 bad_vwgt_length"},
    {"kind": "matching", "mode": "shem", "graph": "star4_w", "seed": 1, "min_matched": 2,
     "ref": "src/coarsen/shem.rs:80-106"},
    {"kind": "matching", "mode": "rm", "graph": "path4", "seed": 42, "min_matched": 2,
     "ref": "src/coarsen/rm.rs:56-64"},
    {"kind": "matching", "mode": "rm", "graph": "path4", "seed": 0, "min_matched": 2,
     "ref": "src/coarsen/rm.rs:66-74"},
    {"kind": "refine_no_increase", "rtype": "greedy", "graph": "cycle4", "part": [0, 1, 0, 1], "nparts": 2,
     "tpwgts": [2.0, 2.0], "ubvec": [1.03], "niter": 10, "ref": "src/refine/greedy.rs:229-239"},
    {"kind": "refine_no_increase", "rtype": "fm", "graph": "grid3x3", "part": [0, 0, 0, 1, 1, 1, 2, 2, 2],
     "nparts": 3, "tpwgts": [3.0, 3.0, 3.0], "ubvec": [1.1], "niter": 5, "ref": "src/refine/fm_kway.rs:209-219"},
]


def main():
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump({"source": "known answers of the reference's unit tests (javagg/rmetis), with file:line",
                   "graphs": GRAPHS, "cases": CASES}, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
