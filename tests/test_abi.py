"""CPU checks of the drop-in boundary: the library loads, exports every
function the public headers declare, and lays out the ABI structs exactly as
Teide's td.h does (offsets committed in tests/golden/abi_layout.json, taken
from the reference header by tests/golden/make_abi_layout.py)."""
import ctypes
import json
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")


def declared(header):
    text = open(os.path.join(INC, header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set()
    for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b((?:td|tdg)_\w+)\s*\(", text, flags=re.M):
        line = text[m.start():m.end()]
        if "static" in line or "#define" in line:
            continue
        names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    import teide_b200
    lib = ctypes.CDLL(teide_b200.lib_path())
    missing = []
    for h in ("teide/td.h", "teide/td_b200.h", "tdg.h"):
        for name in sorted(declared(h)):
            if not hasattr(lib, name):
                missing.append((h, name))
    assert not missing, missing
    assert len(declared("tdg.h")) >= 18


LAYOUT_PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "teide/td.h"
#define O(T, f) printf("\"%s.%s\": %zu,\n", #T, #f, offsetof(T, f))
int main(void) {
    printf("{\n");
    O(td_t, nullmap); O(td_t, mmod); O(td_t, order); O(td_t, type); O(td_t, attrs);
    O(td_t, rc); O(td_t, len); O(td_t, i64); O(td_t, data); O(td_t, slice_offset); O(td_t, sym_dict);
    O(td_op_t, opcode); O(td_op_t, arity); O(td_op_t, flags); O(td_op_t, out_type); O(td_op_t, pad);
    O(td_op_t, id); O(td_op_t, est_rows); O(td_op_t, inputs);
    O(td_op_ext_t, literal); O(td_op_ext_t, keys); O(td_op_ext_t, n_keys); O(td_op_ext_t, n_aggs);
    O(td_op_ext_t, agg_ops); O(td_op_ext_t, agg_ins); O(td_op_ext_t, join.left_keys);
    O(td_op_ext_t, join.right_keys); O(td_op_ext_t, join.n_join_keys); O(td_op_ext_t, join.join_type);
    O(td_op_ext_t, sort.n_cols); O(td_op_ext_t, window.frame_end_n);
    O(td_graph_t, nodes); O(td_graph_t, node_count); O(td_graph_t, node_cap); O(td_graph_t, table);
    O(td_graph_t, tables); O(td_graph_t, n_tables); O(td_graph_t, ext_nodes); O(td_graph_t, ext_count);
    O(td_graph_t, ext_cap); O(td_graph_t, selection);
    O(td_sel_meta_t, total_pass); O(td_sel_meta_t, n_segs);
    O(td_mem_stats_t, sys_peak);
    printf("\"sizeof.td_t\": %zu, \"sizeof.td_op_t\": %zu, \"sizeof.td_op_ext_t\": %zu,\n",
           sizeof(td_t), sizeof(td_op_t), sizeof(td_op_ext_t));
    printf("\"sizeof.td_graph_t\": %zu, \"sizeof.td_sel_meta_t\": %zu, \"sizeof.td_morsel_t\": %zu,\n",
           sizeof(td_graph_t), sizeof(td_sel_meta_t), sizeof(td_morsel_t));
    printf("\"const.OP_GROUP\": %d, \"const.OP_JOIN\": %d, \"const.OP_FILTER\": %d, \"const.OP_AVG\": %d,\n",
           OP_GROUP, OP_JOIN, OP_FILTER, OP_AVG);
    printf("\"const.TD_SEL\": %d, \"const.TD_SYM\": %d, \"const.TD_ERR_CANCEL\": %d, \"const.TD_TYPE_COUNT\": %d\n",
           TD_SEL, TD_SYM, (int)TD_ERR_CANCEL, TD_TYPE_COUNT);
    printf("}\n");
    return 0;
}
"""


def layout_of(include_dir):
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(src, "w").write(LAYOUT_PROBE)
        subprocess.run(["gcc", "-std=c17", "-I", include_dir, src, "-o", exe], check=True)
        return json.loads(subprocess.run([exe], check=True, capture_output=True, text=True).stdout)


def test_struct_layout_matches_teide():
    want = json.load(open(os.path.join(ROOT, "tests", "golden", "abi_layout.json")))
    got = layout_of(INC)
    assert got == want


def test_device_abi_constants_match_header():
    """The kernels hard-code td.h's type tags and opcodes."""
    src = open(os.path.join(ROOT, "teide_b200", "csrc", "cuda", "tdg_common.cuh")).read()
    td_h = open(os.path.join(INC, "teide", "td.h")).read()
    pairs = {"T_I64": "TD_I64", "T_F64": "TD_F64", "T_SYM": "TD_SYM", "T_I32": "TD_I32",
             "T_BOOL": "TD_BOOL", "T_TIMESTAMP": "TD_TIMESTAMP", "A_SUM": "OP_SUM",
             "A_COUNT": "OP_COUNT", "A_AVG": "OP_AVG", "A_MIN": "OP_MIN", "A_MAX": "OP_MAX"}
    for dev, host in pairs.items():
        dv = int(re.search(rf"\b{dev}\s*=\s*(\d+)", src).group(1))
        hv = int(re.search(rf"#define\s+{host}\s+(\d+)", td_h).group(1))
        assert dv == hv, (dev, host)
