"""Builds the in-tree native code: the CUDA library (sm_100a) and, when asked, the CPU oracles
used by the tests (oracle/Makefile). Oracle A is built only when a reference tree is given, as
the `reference` argument or the MP_REFERENCE_TREE environment variable."""
from __future__ import annotations

import os
import subprocess
from typing import Optional

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build_library() -> None:
    subprocess.run(["make", "-j", str(max(1, min(os.cpu_count() or 1, 12))), "-C", os.path.join(HERE, "csrc"),
                    os.path.join(HERE, "libmpgpu.so"),
                    os.path.join(HERE, "libmpgpu_dropin.so")], check=True)


def build_oracles(reference: Optional[str] = None) -> None:
    reference = reference or os.environ.get("MP_REFERENCE_TREE")
    targets = ["oracle-b"]
    args = []
    if reference and os.path.isdir(os.path.join(reference, "impl")):
        targets.append("reference")
        args.append(f"REF={reference}")
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")] + args + targets, check=True)


def build(with_oracles: bool = True, reference: Optional[str] = None) -> None:
    build_library()
    if with_oracles:
        build_oracles(reference)
