"""Write tests/golden/abi_layout.json: field offsets and sizes of the td.h ABI
structs, compiled against Teide's own header (the reference checkout).

    python tests/golden/make_abi_layout.py path/to/reference/include
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from test_abi import layout_of  # noqa: E402

if len(sys.argv) != 2:
    sys.exit("usage: make_abi_layout.py path/to/reference/include")
inc = sys.argv[1]
json.dump(layout_of(inc), open(os.path.join(HERE, "abi_layout.json"), "w"), indent=1, sort_keys=True)
print("wrote", os.path.join(HERE, "abi_layout.json"))
