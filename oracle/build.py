"""Build recipe for the CPU oracle extension (test infrastructure only).

Compiles ``oracle/oracle_py.cpp`` (which includes ``ando_oracle.hpp``) into the
Python extension ``oracle/ando_oracle*.so`` with g++. The product package never
imports it; tests, ``__graft_entry__.smoke`` and ``bench.py``'s CPU-baseline leg do.
"""
from __future__ import annotations

import os
import subprocess
import sys
import sysconfig
from pathlib import Path

HERE = Path(__file__).resolve().parent


def ext_path() -> Path:
    suffix = sysconfig.get_config_var("EXT_SUFFIX") or ".so"
    return HERE / f"ando_oracle{suffix}"


def build(force: bool = False, verbose: bool = False) -> Path:
    out = ext_path()
    srcs = [HERE / "oracle_py.cpp", HERE / "ando_oracle.hpp"]
    if out.exists() and not force and all(out.stat().st_mtime >= s.stat().st_mtime for s in srcs):
        return out
    import pybind11

    cmd = [
        os.environ.get("CXX", "g++"), "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", "-pthread",
        f"-I{pybind11.get_include()}", f"-I{sysconfig.get_paths()['include']}", f"-I{HERE}",
        str(HERE / "oracle_py.cpp"), "-o", str(out) + ".tmp",
    ]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(str(out) + ".tmp", out)
    return out


def load():
    """Import the oracle extension, building it first if needed."""
    build()
    if str(HERE) not in sys.path:
        sys.path.insert(0, str(HERE))
    import ando_oracle  # noqa: E402

    return ando_oracle


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
