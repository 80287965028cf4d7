"""Builds the in-tree native code: the CUDA library (sm_100a) and, when asked, the CPU oracles
used by the tests (oracle/Makefile; Oracle A only where the reference tree is present)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build_library() -> None:
    subprocess.run(["make", "-C", os.path.join(HERE, "csrc"), os.path.join(HERE, "libmpgpu.so"),
                    os.path.join(HERE, "libmpgpu_dropin.so")], check=True)


def build_oracles(reference: str = "/root/reference") -> None:
    targets = ["oracle-b"]
    if os.path.isdir(os.path.join(reference, "impl")):
        targets.append("reference")
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), f"REF={reference}"] + targets, check=True)


def build(with_oracles: bool = True) -> None:
    build_library()
    if with_oracles:
        build_oracles()
