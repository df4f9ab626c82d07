"""teide_b200: a B200-native executor for Teide's relational hot path.

The product is libteide_b200.so, built in-tree from teide_b200/csrc: the C17
host runtime behind include/teide/td.h and the sm_100a kernels behind
include/tdg.h.  This package builds and binds it:

    import teide_b200
    td = teide_b200.load()          # Td binding of libteide_b200.so
    t = td.table({"k": keys, "v": vals})
    g = td.graph(t); ...; res = g.execute(root)

There is no CPU execution path: without a CUDA device td_execute returns
TD_ERR_IO, and without the built library load() raises.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libteide_b200.so")

_td = None


def build(jobs: int = 8) -> str:
    """Compile libteide_b200.so (sm_100a kernels + host runtime) in place."""
    subprocess.run(["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"], check=True,
                   stdout=subprocess.DEVNULL)
    return LIB_PATH


def lib_path() -> str:
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(
            f"{LIB_PATH} is not built; run teide_b200.build() or make -C teide_b200/csrc")
    return LIB_PATH


def load():
    """The Td binding of libteide_b200.so (process-wide singleton)."""
    global _td
    if _td is None:
        from .td import Td
        _td = Td(lib_path())
    return _td


def device_abi():
    """The binding of the device-path C ABI (include/tdg.h)."""
    from .tdg import Tdg
    return Tdg(load().lib)
